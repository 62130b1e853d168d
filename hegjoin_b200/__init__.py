"""hegjoin_b200 -- B200-native epsilon self-join (HEGJoin algorithm 0 drop-in).

Python mirror of the reference's GPU-only join interface over the C ABI in
``include/hegjoin_b200.h`` (libhegjoin_b200.so).  The reference's C++ entry
points map one to one:

    generateNDGridDimensions   (main.cu:449-520)      -> grid_geometry
    gridIndexingGPU            (GPU.cu:74-398)        -> gridIndexingGPU / GridIndex
    sortByWorkLoad             (SortByWorkload.cu:19) -> sortByWorkLoad / GridIndex.sort_by_workload
    distanceTableNDGridBatches (GPU.cu:787-1702)      -> distanceTableNDGridBatches / join

Device buffers are torch CUDA tensors; torch supplies memory and streams only.
All compute runs in the CUDA library; there is no CPU fallback: if the shared
library is missing, importing this package raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhegjoin_b200.so")

HJ_OK = 0
HJ_ERR_INVALID = 1
HJ_ERR_CUDA = 2
HJ_ERR_OOM = 3
HJ_ERR_OVERFLOW = 4
HJ_ERR_TIMEOUT = 5
HJ_ERR_UNSUPPORTED = 6
HJ_ERR_NO_DEVICE = 7
HJ_F32 = 0
HJ_F64 = 1
HJ_REFINE_AUTO = 0
HJ_REFINE_EXACT = 1
HJ_REFINE_TC_F16 = 2
HJ_REFINE_TC_BF16 = 3
REFINE_NAMES = {"auto": 0, "exact": 1, "tc_f16": 2, "tc_bf16": 3}


class HJError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"hegjoin_b200 status {status}: {msg}")
        self.status = status


class IndexInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("d", ctypes.c_uint32), ("k", ctypes.c_uint32), ("dtype", ctypes.c_uint32),
                ("n_nonempty_cells", ctypes.c_uint32), ("grid_aliasing", ctypes.c_uint32),
                ("total_cells", ctypes.c_uint64), ("total_candidates", ctypes.c_uint64),
                ("eps", ctypes.c_double), ("sq_threshold", ctypes.c_double),
                ("min_arr", ctypes.c_double * 16), ("n_cells", ctypes.c_uint32 * 16)]


class JoinOpts(ctypes.Structure):
    _fields_ = [("refine", ctypes.c_int), ("result_capacity", ctypes.c_uint64), ("sample_rate", ctypes.c_double),
                ("mem_fraction", ctypes.c_double), ("query_block", ctypes.c_uint32), ("max_batches", ctypes.c_uint32),
                ("use_graphs", ctypes.c_uint32), ("keep_keys", ctypes.c_uint32), ("shard_count", ctypes.c_uint32),
                ("shard_index", ctypes.c_uint32), ("device_bytes_cap", ctypes.c_uint64),
                ("stream_overlap", ctypes.c_uint32)]


class JoinStats(ctypes.Structure):
    _fields_ = [("total_pairs", ctypes.c_uint64), ("n_batches", ctypes.c_uint32), ("n_retries", ctypes.c_uint32),
                ("band_pairs", ctypes.c_uint64), ("tc_accepts", ctypes.c_uint64), ("estimated_pairs", ctypes.c_uint64),
                ("filter_delta", ctypes.c_double), ("ms_estimate", ctypes.c_float), ("ms_refine", ctypes.c_float),
                ("ms_group", ctypes.c_float), ("ms_total", ctypes.c_float), ("ms_refine_kernel", ctypes.c_float),
                ("refine_launches", ctypes.c_uint32), ("refine_used", ctypes.c_uint32),
                ("kernel_launches", ctypes.c_uint32), ("ms_setup", ctypes.c_float), ("bytes_wanted", ctypes.c_uint64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchView(ctypes.Structure):
    _fields_ = [("batch", ctypes.c_uint32), ("pad_", ctypes.c_uint32), ("count", ctypes.c_uint64),
                ("d_keys", ctypes.c_void_p), ("d_vals", ctypes.c_void_p), ("release_event", ctypes.c_void_p)]


# hj_batch_sink: hj_status (*)(const hj_batch_view*, void* user, void* stream)
BATCH_SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.POINTER(BatchView), ctypes.c_void_p, ctypes.c_void_p)


class Peaks(ctypes.Structure):
    _fields_ = [("fp32_fma_tflops", ctypes.c_double), ("fp32x2_fma_tflops", ctypes.c_double),
                ("fp64_fma_tflops", ctypes.c_double), ("f16_mma_tflops", ctypes.c_double),
                ("bf16_mma_tflops", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_uint64), ("workers", ctypes.c_uint32), ("refine", ctypes.c_int)]


class ServeInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double), ("stats", JoinStats), ("reserved_bytes", ctypes.c_uint64),
                ("regrants", ctypes.c_uint32)]


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C hegjoin_b200/csrc` "
                          "(or __graft_entry__.build()); there is no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    P, U32, U64, I, D = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
    sigs = {
        "hj_last_error": (ctypes.c_char_p, []),
        "hj_version": (ctypes.c_char_p, []),
        "hj_kernel_launch_count": (U64, []),
        "hj_grid_geometry": (I, [P, U32, U32, U32, I, D, P, P, P, P, P]),
        "hj_index_create": (I, [P, U32, U32, U32, I, D, P, P, P, P]),
        "hj_index_destroy": (I, [P]),
        "hj_index_get_info": (I, [P, P]),
        "hj_index_export": (I, [P, P, P, P, P]),
        "hj_index_views": (I, [P, P, P, P, P]),
        "hj_sort_by_workload": (I, [P, P, P]),
        "hj_workload_export": (I, [P, P, P, P]),
        "hj_join_opts_default": (None, [P]),
        "hj_join": (I, [P, P, P, P, P]),
        "hj_result_destroy": (I, [P]),
        "hj_result_num_batches": (I, [P, P, P]),
        "hj_result_batch": (I, [P, U32, P, P, P]),
        "hj_result_table": (I, [P, P]),
        "hj_result_to_csr": (I, [P, P, P, I, P]),
        "hj_result_digest": (I, [P, P, P, P, P]),
        "hj_self_join_host": (I, [P, U32, U32, U32, I, D, P, P, P, P]),
        "hj_probe_sqdist": (I, [P, P, U32, U32, I, P, P]),
        "hj_probe_tc_tile": (I, [P, I, U32, U32, P, P, P, P]),
        "hj_tc_operand_scale": (I, [P, P]),
        "hj_probe_tc_wait_timeout": (I, [P, I, U64, P]),
        "hj_shard_plan": (I, [U32, U32, U32, P, P, P]),
        "hj_shard_plan_lpt": (I, [P, U32, U32, U32, P, P]),
        "hj_join_stream": (I, [P, P, BATCH_SINK, P, P, P, P, P, P]),
        "hj_debug_fail_alloc": (None, [U64]),
        "hj_measure_peaks": (I, [P, P]),
        "hj_debug_pool_used": (I, [P]),
        "hj_debug_pool_peak": (I, [P, I]),
        "hj_import_text": (I, [ctypes.c_char_p, U32, I, P, P]),
        "hj_import_binary": (I, [ctypes.c_char_p, U32, I, P, P]),
        "hj_write_binary": (I, [ctypes.c_char_p, P, U64, U32, I]),
        "hj_host_free": (None, [P]),
        "hj_server_opts_default": (None, [P]),
        "hj_server_create": (I, [P, P]),
        "hj_server_submit": (I, [P, P, U32, U32, U32, I, D, P]),
        "hj_server_wait": (I, [P, U64, D, P, P]),
        "hj_server_destroy": (I, [P]),
        "hj_server_usage": (I, [P, P, P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def last_error() -> str:
    return (lib.hj_last_error() or b"").decode()


def check(status: int) -> None:
    if status != HJ_OK:
        raise HJError(status, last_error())


def kernel_launch_count() -> int:
    return int(lib.hj_kernel_launch_count())


def _torch():
    import torch
    return torch


def _stream_ptr(stream) -> int | None:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None


def _dtype_code(t) -> int:
    torch = _torch()
    if t.dtype == torch.float32:
        return HJ_F32
    if t.dtype == torch.float64:
        return HJ_F64
    raise ValueError(f"unsupported dataset dtype {t.dtype} (float32 or float64)")


def _ptr(t) -> int:
    return t.data_ptr()


def grid_geometry(db, k: int, eps: float, stream=None):
    """generateNDGridDimensions (main.cu:449-520): (minArr, maxArr, nCells, totalCells)."""
    n, d = db.shape
    mn = (ctypes.c_double * k)()
    mx = (ctypes.c_double * k)()
    nc = (ctypes.c_uint32 * k)()
    tot = ctypes.c_uint64()
    check(lib.hj_grid_geometry(_ptr(db), n, d, k, _dtype_code(db), float(eps), mn, mx, nc, ctypes.byref(tot),
                               _stream_ptr(stream)))
    return list(mn), list(mx), list(nc), int(tot.value)


class GridIndex:
    """Device grid index over an n x d dataset (gridIndexingGPU, GPU.cu:74-398)."""

    def __init__(self, db, k: int, eps: float, min_arr=None, n_cells=None, stream=None):
        torch = _torch()
        if not db.is_cuda or not db.is_contiguous():
            raise ValueError("db must be a contiguous CUDA tensor")
        self.db = db
        n, d = db.shape
        self._stream = stream
        h = ctypes.c_void_p()
        mn = (ctypes.c_double * k)(*min_arr) if min_arr is not None else None
        nc = (ctypes.c_uint32 * k)(*n_cells) if n_cells is not None else None
        check(lib.hj_index_create(_ptr(db), n, d, k, _dtype_code(db), float(eps), mn, nc, _stream_ptr(stream),
                                  ctypes.byref(h)))
        self._h = h
        self.torch = torch

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.hj_index_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self) -> IndexInfo:
        inf = IndexInfo()
        check(lib.hj_index_get_info(self._h, ctypes.byref(inf)))
        return inf

    def export(self):
        """(gridCellLookup linear ids, grid indexmin, grid indexmax, indexLookupArr) as CUDA tensors."""
        torch = self.torch
        inf = self.info()
        nc, n = inf.n_nonempty_cells, inf.n
        lookup = torch.empty((max(nc, 1), 2), dtype=torch.int64, device=self.db.device)
        grid = torch.empty((max(nc, 1), 2), dtype=torch.int32, device=self.db.device)
        ilu = torch.empty(n, dtype=torch.int32, device=self.db.device)
        check(lib.hj_index_export(self._h, _ptr(lookup), _ptr(grid), _ptr(ilu), _stream_ptr(self._stream)))
        idx = (lookup[:nc, 0] & 0xFFFFFFFF)
        return lookup[:nc, 1], grid[:nc, 0], grid[:nc, 1], ilu, idx

    def views(self):
        pts = ctypes.c_void_p(); perm = ctypes.c_void_p(); lid = ctypes.c_void_p(); cs = ctypes.c_void_p()
        check(lib.hj_index_views(self._h, ctypes.byref(pts), ctypes.byref(perm), ctypes.byref(lid), ctypes.byref(cs)))
        return pts.value, perm.value, lid.value, cs.value

    def sort_by_workload(self) -> int:
        tot = ctypes.c_uint64()
        check(lib.hj_sort_by_workload(self._h, _stream_ptr(self._stream), ctypes.byref(tot)))
        return int(tot.value)

    def workload_export(self):
        """(schedulingCell[nNonEmpty] as (nbPoints, cellId) int32 pairs, originPointIndex[n])."""
        torch = self.torch
        inf = self.info()
        sched = torch.empty((max(inf.n_nonempty_cells, 1), 2), dtype=torch.int32, device=self.db.device)
        origin = torch.empty(inf.n, dtype=torch.int32, device=self.db.device)
        check(lib.hj_workload_export(self._h, _ptr(sched), _ptr(origin), _stream_ptr(self._stream)))
        return sched[:inf.n_nonempty_cells], origin


class JoinResult:
    """Device result of a join: per-batch neighbour ids grouped by query, plus the neighbour table."""

    def __init__(self, handle, stats: JoinStats, n: int, device):
        self._h = handle
        self.stats = stats
        self.n = n
        self.device = device

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.hj_result_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def total_pairs(self) -> int:
        return int(self.stats.total_pairs)

    def to_csr(self, sort_lists: bool = True, stream=None):
        torch = _torch()
        off = torch.empty(self.n + 1, dtype=torch.int64, device=self.device)
        vals = torch.empty(max(self.total_pairs, 1), dtype=torch.int32, device=self.device)
        check(lib.hj_result_to_csr(self._h, _ptr(off), _ptr(vals), int(sort_lists), _stream_ptr(stream)))
        return off, vals[:self.total_pairs]

    def digest(self, stream=None):
        torch = _torch()
        cnt = torch.empty(self.n, dtype=torch.int32, device=self.device)
        s = torch.empty(self.n, dtype=torch.int64, device=self.device)
        x = torch.empty(self.n, dtype=torch.int64, device=self.device)
        check(lib.hj_result_digest(self._h, _ptr(cnt), _ptr(s), _ptr(x), _stream_ptr(stream)))
        return cnt, s, x

    def batches(self):
        nb = ctypes.c_uint32(); tot = ctypes.c_uint64()
        check(lib.hj_result_num_batches(self._h, ctypes.byref(nb), ctypes.byref(tot)))
        out = []
        for b in range(nb.value):
            v = ctypes.c_void_p(); k = ctypes.c_void_p(); c = ctypes.c_uint64()
            check(lib.hj_result_batch(self._h, b, ctypes.byref(v), ctypes.byref(k), ctypes.byref(c)))
            out.append((v.value, k.value, int(c.value)))
        return out

    def table_ptr(self) -> int:
        t = ctypes.c_void_p()
        check(lib.hj_result_table(self._h, ctypes.byref(t)))
        return t.value


def join_opts(refine="auto", result_capacity=0, sample_rate=0.0, mem_fraction=0.0, max_batches=0,
              use_graphs=False, keep_keys=False, shard_count=0, shard_index=0, device_bytes_cap=0,
              stream_overlap=False) -> JoinOpts:
    o = JoinOpts()
    lib.hj_join_opts_default(ctypes.byref(o))
    o.refine = REFINE_NAMES[refine] if isinstance(refine, str) else int(refine)
    o.result_capacity = int(result_capacity)
    if sample_rate:
        o.sample_rate = float(sample_rate)
    if mem_fraction:
        o.mem_fraction = float(mem_fraction)
    o.max_batches = int(max_batches)
    o.use_graphs = int(bool(use_graphs))
    o.keep_keys = int(bool(keep_keys))
    o.shard_count = int(shard_count)
    o.shard_index = int(shard_index)
    o.device_bytes_cap = int(device_bytes_cap)
    o.stream_overlap = int(bool(stream_overlap))
    return o


def join(index: GridIndex, stream=None, **kw) -> JoinResult:
    """distanceTableNDGridBatches (GPU.cu:787-1702) for algorithm 0, result kept on the device."""
    o = join_opts(**kw)
    st = JoinStats()
    h = ctypes.c_void_p()
    status = lib.hj_join(index.handle, ctypes.byref(o), _stream_ptr(stream), ctypes.byref(h), ctypes.byref(st))
    if status != HJ_OK:
        err = HJError(status, last_error())
        err.stats = st          # what the join knew (bytes_wanted when its cap refused it)
        raise err
    return JoinResult(h, st, index.info().n, index.db.device)


def join_stream(index: GridIndex, sink=None, digest: bool = True, stream=None, **kw):
    """The join with nothing kept on the device (hj_join_stream): every grouped batch
    goes to `sink(batch, count, keys_ptr, vals_ptr, stream_ptr)` (device pointers,
    valid for work enqueued on that stream) and per-query digests accumulate on the
    device.  With stream_overlap=True the sink may instead read the batch on a stream
    of its own and return (status, event_handle): a raw cudaEvent_t recorded after
    those reads (e.g. torch.cuda.Event().cuda_event), kept alive until the join
    returns.  Returns (JoinStats, (count, sum, xor) CUDA tensors or None)."""
    torch = _torch()
    n = index.info().n
    dev = index.db.device
    cnt = s = x = None
    if digest:
        cnt = torch.empty(n, dtype=torch.int32, device=dev)
        s = torch.empty(n, dtype=torch.int64, device=dev)
        x = torch.empty(n, dtype=torch.int64, device=dev)
    errors = []

    def _cb(view, user, st):
        try:
            v = view.contents
            r = sink(int(v.batch), int(v.count), v.d_keys, v.d_vals, st)
            if isinstance(r, tuple):
                r, ev = r
                view.contents.release_event = ev
            return HJ_OK if r is None else int(r)
        except Exception as e:          # a Python error stops the join with a clear status
            errors.append(e)
            return HJ_ERR_INVALID

    cb = BATCH_SINK(_cb) if sink is not None else BATCH_SINK()
    o = join_opts(**kw)
    st = JoinStats()
    status = lib.hj_join_stream(index.handle, ctypes.byref(o), cb, None, _ptr(cnt) if digest else None,
                                _ptr(s) if digest else None, _ptr(x) if digest else None, _stream_ptr(stream),
                                ctypes.byref(st))
    if errors:
        raise errors[0]
    check(status)
    return st, ((cnt, s, x) if digest else None)


def shard_plan_lpt(costs, shard_count: int, shard_index: int) -> np.ndarray:
    """Item indices (ascending) that rank `shard_index` takes under greedy LPT."""
    c = np.ascontiguousarray(costs, dtype=np.uint64)
    items = np.zeros(max(1, len(c)), np.uint32)
    m = ctypes.c_uint32()
    check(lib.hj_shard_plan_lpt(c.ctypes.data, len(c), shard_count, shard_index, items.ctypes.data, ctypes.byref(m)))
    return items[:m.value]


def measure_peaks(stream=None) -> dict:
    """This library's own measured pipe peaks in TFLOP/s (hj_measure_peaks)."""
    p = Peaks()
    check(lib.hj_measure_peaks(ctypes.byref(p), _stream_ptr(stream)))
    return p.as_dict()


def debug_fail_alloc(nth: int) -> None:
    """Make the nth device allocation from now fail as an out-of-memory would (0 disarms)."""
    lib.hj_debug_fail_alloc(int(nth))


def debug_pool_used() -> int:
    b = ctypes.c_uint64()
    check(lib.hj_debug_pool_used(ctypes.byref(b)))
    return int(b.value)


def debug_pool_peak(reset: bool = False) -> int:
    """Most bytes the library's memory pool held since the last reset."""
    b = ctypes.c_uint64()
    check(lib.hj_debug_pool_peak(ctypes.byref(b), int(bool(reset))))
    return int(b.value)


def self_join_host(db: np.ndarray, k: int, eps: float, stream=None, keep=True, **kw):
    """One-shot join from host memory (copies in, index, workload order, join)."""
    db = np.ascontiguousarray(db)
    dt = HJ_F32 if db.dtype == np.float32 else HJ_F64
    o = join_opts(**kw)
    st = JoinStats()
    h = ctypes.c_void_p()
    check(lib.hj_self_join_host(db.ctypes.data, db.shape[0], db.shape[1], k, dt, float(eps), ctypes.byref(o),
                                _stream_ptr(stream), ctypes.byref(h) if keep else None, ctypes.byref(st)))
    torch = _torch()
    return JoinResult(h if keep else ctypes.c_void_p(), st, db.shape[0], torch.device("cuda"))


# ---- names of the reference's entry points ---------------------------------------------
def gridIndexingGPU(db, k: int, eps: float, min_arr=None, n_cells=None, stream=None) -> GridIndex:
    return GridIndex(db, k, eps, min_arr, n_cells, stream)


def sortByWorkLoad(index: GridIndex) -> int:
    return index.sort_by_workload()


def distanceTableNDGridBatches(index: GridIndex, **kw) -> JoinResult:
    return join(index, **kw)


def probe_sqdist(a, b, stream=None):
    """Evaluate kernel.cu:350-353's expression as nvcc compiles it by default (row-wise pairs)."""
    torch = _torch()
    n, d = a.shape
    out = torch.empty(n, dtype=a.dtype, device=a.device)
    check(lib.hj_probe_sqdist(_ptr(a), _ptr(b), n, d, _dtype_code(a), _ptr(out), _stream_ptr(stream)))
    return out


def shard_plan(n_items: int, shard_count: int, shard_index: int):
    """(first, stride, count) of the work items rank `shard_index` processes."""
    f, s, m = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    check(lib.hj_shard_plan(n_items, shard_count, shard_index, ctypes.byref(f), ctypes.byref(s), ctypes.byref(m)))
    return f.value, s.value, m.value


def _take_host(ptr: ctypes.c_void_p, n: int, d: int, dtype) -> np.ndarray:
    """Copy a library-allocated n x d host array into numpy and release it."""
    try:
        if n == 0:
            return np.zeros((0, d), dtype=dtype)
        buf = (ctypes.c_char * (n * d * np.dtype(dtype).itemsize)).from_address(ptr.value)
        return np.frombuffer(buf, dtype=dtype).reshape(n, d).copy()
    finally:
        lib.hj_host_free(ptr)


def import_text(path: str, d: int, dtype=np.float32) -> np.ndarray:
    """importNDDataset (import_dataset.cpp:10-40): the reference's text format, parsed in parallel."""
    out, n = ctypes.c_void_p(), ctypes.c_uint64()
    check(lib.hj_import_text(os.fsencode(path), d, HJ_F32 if np.dtype(dtype) == np.float32 else HJ_F64,
                             ctypes.byref(out), ctypes.byref(n)))
    return _take_host(out, n.value, d, dtype)


def import_binary(path: str, d: int, dtype=np.float32) -> np.ndarray:
    """The binary twin (or the reference's raw binary layout)."""
    out, n = ctypes.c_void_p(), ctypes.c_uint64()
    check(lib.hj_import_binary(os.fsencode(path), d, HJ_F32 if np.dtype(dtype) == np.float32 else HJ_F64,
                               ctypes.byref(out), ctypes.byref(n)))
    return _take_host(out, n.value, d, dtype)


def write_binary(path: str, db: np.ndarray) -> None:
    db = np.ascontiguousarray(db)
    check(lib.hj_write_binary(os.fsencode(path), db.ctypes.data, db.shape[0], db.shape[1],
                              HJ_F32 if db.dtype == np.float32 else HJ_F64))


def generate_exp40(seed: int, n: int, d: int, dtype=np.float32, stream: int = 0) -> np.ndarray:
    """Host generator (C++/OpenMP, libhj_datagen.so): the values of workloads.exp40."""
    from . import workloads
    return workloads.exp40(seed, n, d, dtype, stream)


def generate_skewed(seed: int, n: int, d: int, n_clusters: int = 64, sigma: float = 0.002,
                    frac_clustered: float = 0.2, dtype=np.float32) -> np.ndarray:
    """Host generator of the skewed workload (80% Exp(40), 20% Gaussian clusters)."""
    from . import workloads
    return workloads.skewed(seed, n, d, n_clusters, sigma, frac_clustered, dtype)


class _DeviceArray:
    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_view(ptr: int, shape, dtype):
    """A torch tensor over library-owned device memory (no copy; valid while the owner lives)."""
    torch = _torch()
    typestr = {np.float32: "<f4", np.float64: "<f8", np.uint32: "<u4", np.int32: "<i4",
               np.uint64: "<u8", np.int64: "<i8"}[np.dtype(dtype).type]
    return torch.as_tensor(_DeviceArray(ptr, shape, typestr), device="cuda")


def kpad_for(d: int) -> int:
    return ((d + 4 + 31) // 32) * 32


def probe_tc_tile(index: GridIndex, refine: str, a0: int, b0: int, stream=None):
    """One candidate tile x 512 queries through the tensor-core path.

    Returns (accumulators [128, 512], query-form rows [512, kpad], candidate-form
    rows [128, kpad]) as float64 numpy arrays in the dataset's units: the
    filter's power-of-two operand scale is divided out exactly.
    """
    torch = _torch()
    inf = index.info()
    kp = kpad_for(inf.d)
    out = torch.empty((128, 512), dtype=torch.float32, device=index.db.device)
    hq = np.zeros((512, kp), np.uint16)
    hc = np.zeros((128, kp), np.uint16)
    check(lib.hj_probe_tc_tile(index.handle, REFINE_NAMES[refine], a0, b0, _ptr(out), hq.ctypes.data,
                               hc.ctypes.data, _stream_ptr(stream)))
    s = ctypes.c_int()
    check(lib.hj_tc_operand_scale(index.handle, ctypes.byref(s)))
    # the operand forms hold (x - min) * 2^s: return everything in the dataset's units
    # (power-of-two scaling is exact)
    if refine == "tc_bf16":
        conv = lambda a: np.ldexp((a.astype(np.uint32) << 16).view(np.float32).astype(np.float64), -s.value)
    else:
        conv = lambda a: np.ldexp(a.view(np.float16).astype(np.float64), -s.value)
    acc = np.ldexp(out.cpu().numpy().astype(np.float64), -2 * s.value)
    return acc, conv(hq), conv(hc)


class Server:
    """Continuous-batching join service (hj_server_*): submit host datasets, wait for device results."""

    def __init__(self, workers: int = 4, hbm_budget: int = 150 << 30, refine="auto"):
        o = ServerOpts()
        lib.hj_server_opts_default(ctypes.byref(o))
        o.workers = workers
        o.hbm_budget = hbm_budget
        o.refine = REFINE_NAMES[refine] if isinstance(refine, str) else int(refine)
        self._h = ctypes.c_void_p()
        check(lib.hj_server_create(ctypes.byref(o), ctypes.byref(self._h)))
        self._keep = {}

    def submit(self, db: np.ndarray, k: int, eps: float) -> int:
        db = np.ascontiguousarray(db)
        t = ctypes.c_uint64()
        check(lib.hj_server_submit(self._h, db.ctypes.data, db.shape[0], db.shape[1], k,
                                   HJ_F32 if db.dtype == np.float32 else HJ_F64, float(eps), ctypes.byref(t)))
        self._keep[t.value] = db          # the host buffer must outlive the request
        return t.value

    def wait(self, ticket: int, keep_result: bool = True, timeout: float = 0.0):
        h = ctypes.c_void_p()
        info = ServeInfo()
        st = lib.hj_server_wait(self._h, ticket, float(timeout), ctypes.byref(h) if keep_result else None,
                                ctypes.byref(info))
        db = self._keep.pop(ticket, None)
        check(st)
        res = None
        if keep_result:
            import torch
            res = JoinResult(h, info.stats, db.shape[0], torch.device("cuda"))
        return res, info

    def usage(self) -> tuple:
        """(bytes held against the budget now, the most ever held)."""
        cur, peak = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib.hj_server_usage(self._h, ctypes.byref(cur), ctypes.byref(peak)))
        return cur.value, peak.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.hj_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
