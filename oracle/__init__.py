"""oracle -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over oracle/_ref/libhj_oracle.so, the CPU restatement of the
reference's algorithm-0 semantics (see hj_oracle.cpp for the file:line of
every rule).  Imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg as the checker; never by the product package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libhj_oracle.so")


def build() -> None:
    subprocess.run(["make", "-C", _HERE], check=True, stdout=subprocess.DEVNULL)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = ctypes.CDLL(LIB_PATH)
    P, U32, U64, I, F, D = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_float,
                            ctypes.c_double)
    for suf, T in (("f32", F), ("f64", D)):
        getattr(lib, f"hjo_geometry_{suf}").argtypes = [P, U32, U32, U32, T, P, P, P, P]
        getattr(lib, f"hjo_geometry_{suf}").restype = None
        getattr(lib, f"hjo_index_{suf}").argtypes = [P, U32, U32, U32, T, P, P, P, P, P, P]
        getattr(lib, f"hjo_index_{suf}").restype = U32
        getattr(lib, f"hjo_cell_workload_{suf}").argtypes = [P, U32, U32, U32, T, P, P, P]
        getattr(lib, f"hjo_cell_workload_{suf}").restype = U64
        getattr(lib, f"hjo_join_{suf}").argtypes = [P, U32, U32, U32, T, P, P, I, P, P, P]
        getattr(lib, f"hjo_join_{suf}").restype = U64
        getattr(lib, f"hjo_join_sample_{suf}").argtypes = [P, U32, U32, U32, T, P, P, P, U32, P]
        getattr(lib, f"hjo_join_sample_{suf}").restype = U64
        getattr(lib, f"hjo_join_lists_{suf}").argtypes = [P, U32, U32, U32, T, P, P, P, U32, P, P, U64]
        getattr(lib, f"hjo_join_lists_{suf}").restype = U64
        getattr(lib, f"hjo_sqdist_{suf}").argtypes = [P, P, U32, I]
        getattr(lib, f"hjo_sqdist_{suf}").restype = D
    for suf in ("f32", "f64"):
        getattr(lib, f"hjo_import_text_{suf}").argtypes = [ctypes.c_char_p, P, U64]
        getattr(lib, f"hjo_import_text_{suf}").restype = U64
    lib.hjo_write_text.argtypes = [ctypes.c_char_p, P, U64, U32, I, I]
    lib.hjo_write_text.restype = I
    lib.hjo_ref_cell_order.argtypes = [P, U32, P]
    lib.hjo_ref_cell_order.restype = None
    lib.hjo_digest.argtypes = [P, P, U32, P, P]
    lib.hjo_digest.restype = None
    lib.hjo_num_threads.restype = I
    return lib


lib = _load()


def _suf(db: np.ndarray) -> str:
    if db.dtype == np.float32:
        return "f32"
    if db.dtype == np.float64:
        return "f64"
    raise ValueError(db.dtype)


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def geometry(db: np.ndarray, k: int, eps):
    """main.cu:449-520: (minArr, maxArr, nCells, totalCells) in the dataset dtype."""
    db = np.ascontiguousarray(db)
    n, d = db.shape
    mn = np.zeros(k, db.dtype)
    mx = np.zeros(k, db.dtype)
    nc = np.zeros(k, np.uint32)
    tot = ctypes.c_uint64()
    getattr(lib, f"hjo_geometry_{_suf(db)}")(_p(db), n, d, k, db.dtype.type(eps), _p(mn), _p(mx), _p(nc),
                                             ctypes.byref(tot))
    return mn, mx, nc, int(tot.value)


def index(db: np.ndarray, k: int, eps, min_arr, n_cells):
    """GPU.cu:74-398: (cell linear ids, grid first, grid last, indexLookupArr)."""
    db = np.ascontiguousarray(db)
    n, d = db.shape
    lid = np.zeros(n, np.uint64)
    first = np.zeros(n, np.int32)
    last = np.zeros(n, np.int32)
    lookup = np.zeros(n, np.uint32)
    mn = np.ascontiguousarray(min_arr, dtype=db.dtype)
    nc = np.ascontiguousarray(n_cells, dtype=np.uint32)
    ncell = getattr(lib, f"hjo_index_{_suf(db)}")(_p(db), n, d, k, db.dtype.type(eps), _p(mn), _p(nc), _p(lid),
                                                  _p(first), _p(last), _p(lookup))
    return lid[:ncell], first[:ncell], last[:ncell], lookup


def cell_workload(db: np.ndarray, k: int, eps, min_arr, n_cells):
    """kernel.cu:74-144: candidates per non-empty cell (cell order) and totalCandidates."""
    db = np.ascontiguousarray(db)
    n, d = db.shape
    nb = np.zeros(n, np.uint32)
    mn = np.ascontiguousarray(min_arr, dtype=db.dtype)
    nc = np.ascontiguousarray(n_cells, dtype=np.uint32)
    tot = getattr(lib, f"hjo_cell_workload_{_suf(db)}")(_p(db), n, d, k, db.dtype.type(eps), _p(mn), _p(nc), _p(nb))
    ncell = len(index(db, k, eps, min_arr, n_cells)[0])
    return nb[:ncell], int(tot)


def join(db: np.ndarray, k: int, eps, min_arr=None, n_cells=None, fma_mode: int = 1, lists: bool = True):
    """kernel.cu:727-802: CSR (offsets[n+1] u64, vals u32) by original query id, lists sorted ascending."""
    db = np.ascontiguousarray(db)
    n, d = db.shape
    if min_arr is None or n_cells is None:
        min_arr, _, n_cells, _ = geometry(db, k, eps)
    mn = np.ascontiguousarray(min_arr, dtype=db.dtype)
    nc = np.ascontiguousarray(n_cells, dtype=np.uint32)
    fn = getattr(lib, f"hjo_join_{_suf(db)}")
    counts = np.zeros(n, np.uint32)
    total = fn(_p(db), n, d, k, db.dtype.type(eps), _p(mn), _p(nc), fma_mode, _p(counts), None, None)
    off = np.zeros(n + 1, np.uint64)
    np.cumsum(counts, out=off[1:])
    if not lists:
        return off, None
    vals = np.zeros(max(total, 1), np.uint32)
    fn(_p(db), n, d, k, db.dtype.type(eps), _p(mn), _p(nc), fma_mode, _p(counts), _p(off), _p(vals))
    return off, vals[:total]


def join_sample(db: np.ndarray, k: int, eps, qids: np.ndarray, min_arr=None, n_cells=None):
    """Pairs emitted by the sampled queries and the seconds the refine took (all OpenMP threads)."""
    db = np.ascontiguousarray(db)
    n, d = db.shape
    if min_arr is None or n_cells is None:
        min_arr, _, n_cells, _ = geometry(db, k, eps)
    mn = np.ascontiguousarray(min_arr, dtype=db.dtype)
    nc = np.ascontiguousarray(n_cells, dtype=np.uint32)
    q = np.ascontiguousarray(qids, dtype=np.uint32)
    sec = ctypes.c_double()
    pairs = getattr(lib, f"hjo_join_sample_{_suf(db)}")(_p(db), n, d, k, db.dtype.type(eps), _p(mn), _p(nc), _p(q),
                                                       len(q), ctypes.byref(sec))
    return int(pairs), float(sec.value)


def join_lists(db: np.ndarray, k: int, eps, qids: np.ndarray, min_arr=None, n_cells=None):
    """Neighbour lists of the sampled query ids: (counts[len(qids)], concatenated sorted lists)."""
    db = np.ascontiguousarray(db)
    n, d = db.shape
    if min_arr is None or n_cells is None:
        min_arr, _, n_cells, _ = geometry(db, k, eps)
    mn = np.ascontiguousarray(min_arr, dtype=db.dtype)
    nc = np.ascontiguousarray(n_cells, dtype=np.uint32)
    q = np.ascontiguousarray(qids, dtype=np.uint32)
    counts = np.zeros(len(q), np.uint32)
    fn = getattr(lib, f"hjo_join_lists_{_suf(db)}")
    cap = max(1, 256 * len(q))
    while True:
        vals = np.zeros(cap, np.uint32)
        total = fn(_p(db), n, d, k, db.dtype.type(eps), _p(mn), _p(nc), _p(q), len(q), _p(counts), _p(vals), cap)
        if total <= cap:
            return counts, vals[:total]
        cap = int(total)


def digest(off: np.ndarray, vals: np.ndarray):
    """Per-query (count, sum of mix64(id), xor of mix64(id ^ salt))."""
    n = len(off) - 1
    off = np.ascontiguousarray(off, dtype=np.uint64)
    vals = np.ascontiguousarray(vals, dtype=np.uint32)
    s = np.zeros(n, np.uint64)
    x = np.zeros(n, np.uint64)
    lib.hjo_digest(_p(off), _p(vals) if len(vals) else None, n, _p(s), _p(x))
    return np.diff(off).astype(np.uint32), s, x


def sqdist(a: np.ndarray, b: np.ndarray, fma_mode: int = 1) -> float:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b, dtype=a.dtype)
    return getattr(lib, f"hjo_sqdist_{_suf(a)}")(_p(a), _p(b), a.shape[-1], fma_mode)


def sq_threshold(eps, dtype) -> float:
    """Largest value x of `dtype` with RN(sqrt(x)) <= eps (numpy's sqrt is IEEE)."""
    t = np.dtype(dtype).type
    e = t(eps)
    x = t(e * e)
    while x > 0 and np.sqrt(x) > e:
        x = np.nextafter(x, t(0))
    while True:
        nx = np.nextafter(x, t(np.inf))
        if np.sqrt(nx) <= e:
            x = nx
        else:
            break
    return x


def ref_cell_order(nb: np.ndarray) -> np.ndarray:
    """The reference's std::sort order of cells by candidate count (SortByWorkload.cu:97-98)."""
    nb = np.ascontiguousarray(nb, dtype=np.uint32)
    out = np.zeros(len(nb), np.int32)
    lib.hjo_ref_cell_order(_p(nb), len(nb), _p(out))
    return out


def ref_batches(counts: np.ndarray, origin: np.ndarray):
    """The reference's batch plan (GPUBatchEst_v2, GPU.cu:403-779) from exact per-query counts.

    `counts` is indexed by original query id, `origin` is originPointIndex.
    Returns (GPUBufferSize, [(first, second)], actual pairs per batch); the
    estimate's unfilled tail is taken as zero.
    """
    n = len(origin)
    n_est = int(n * 0.10)
    r = counts[origin[np.arange(n_est) * 10]].astype(np.int64)
    seqs = n // 10
    full = np.zeros(n, np.int64)
    full_est = 0
    for i in range(seqs - 1):
        m = max(r[i], r[i + 1])
        full[i * 10] = r[i]
        full[i * 10 + 1:(i + 1) * 10] = m
        full_est += r[i] + 9 * m
    buf = 50_000_000
    if full_est < buf * 6:
        buf = full_est // 6
    reserve = int(buf * 0.05)
    batches = []
    b0, run = 0, 0
    for i in range(n):
        run += int(full[i])
        if buf - reserve <= run:
            batches.append((b0, i))
            b0, run = i, 0
        elif i == n - 1:
            batches.append((b0, n))
    per_q = counts[origin].astype(np.int64)
    csum = np.concatenate([[0], np.cumsum(per_q)])
    actual = [int(csum[b] - csum[a]) for a, b in batches]
    return buf, batches, actual


def write_text(path: str, db: np.ndarray, digits: int) -> None:
    """The reference generator's text layout ("v, v, ..., v" lines), `digits` significant digits."""
    db = np.ascontiguousarray(db)
    if lib.hjo_write_text(path.encode(), db.ctypes.data, db.shape[0], db.shape[1], int(db.dtype == np.float64),
                          digits) != 0:
        raise OSError(f"cannot write {path}")


def import_text(path: str, dtype) -> np.ndarray:
    """import_dataset.cpp:10-40 restated: every value the file holds, in order (flat)."""
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    fn = getattr(lib, f"hjo_import_text_{suf}")
    n = fn(path.encode(), None, 0)
    out = np.zeros(max(1, n), dtype=dtype)
    fn(path.encode(), out.ctypes.data, n)
    return out[:n]


def num_threads() -> int:
    return int(lib.hjo_num_threads())
