"""Benchmark: result pairs/s of the epsilon self-join on one workload.

A step is one complete self-join of the workload's dataset: grid index build,
workload order, selectivity estimate, refine and device result table, with the
dataset already resident in HBM (360 MB for the 18-D workload, larger than the
126 MB L2, so no flush is needed between steps).  `e2e` measures the same
metric through the C ABI's host entry point: host->device copy of the dataset
from pinned memory, the join, and a device->host copy of the whole result
(per-query offsets and neighbour ids) into pinned memory, every step.

Multi-GPU (torchrun): every rank holds the dataset and index; the
heaviest-first work items are dealt round robin to ranks (no data-path
collective); value = pairs of all ranks / max-over-ranks step time.

--impl reference times the reference's CPU path on this host's cores on a
bounded query sample (its own build when present, else the CPU restatement).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def peaks():
    try:
        with open(PEAKS_PATH) as f:
            return json.load(f), "measured"
    except Exception:
        return FALLBACK_PEAKS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"hj_clocks_{os.getpid()}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1])); mx.append(float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        if sm:
            out.update(sm_mhz=statistics.median(sm), sm_max_mhz=max(mx), reasons=sorted(reasons), samples=len(sm))
        return out


def dist_init():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def allreduce(vals, op):
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device="cuda")
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=op)
    return t.tolist()


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


# reference build (oracle/ref/Makefile) whose GPUNUMDIM/NUMINDEXEDDIM/DTYPE match each workload
REF_BUILD = {"c2_18d": "c2", "c3_90d": "r90d", "c4_skew6d": "r6d"}


def cpu_baseline(db, wl, seconds_target=20.0):
    """The reference's own CPU join (Super-EGO, Util::egoJoinV2) on a bounded query
    sample against the full dataset, all host cores; the CPU restatement of the
    GPU path when no matching reference build exists."""
    exe = os.path.join(ROOT, "oracle", "_ref", REF_BUILD.get(wl.name, "-"), "ego_driver")
    if os.path.exists(exe):
        path = os.path.join("/tmp", f"hj_{wl.name}_{os.getpid()}.bin")
        with open(path, "wb") as f:
            np.array([db.shape[0], db.shape[1], db.dtype.itemsize], np.uint32).tofile(f)
            db.tofile(f)
        try:
            p = subprocess.run([exe, path, repr(float(wl.eps)), str(seconds_target)], capture_output=True,
                               text=True, timeout=max(600, 20 * seconds_target))
        finally:
            os.unlink(path)
        line = [l for l in p.stdout.splitlines() if l.startswith("HJEGO ")]
        if p.returncode == 0 and line:
            r = json.loads(line[-1][6:])
            return {"value": r["pairs"] / r["seconds"], "unit": "pairs/s", "cores": r["threads"],
                    "kind": "reference",
                    "sample": f"Super-EGO (the reference's CPU join, Util::egoJoinV2) for {r['queries']} evenly "
                              f"spaced query points against all {r['n']} points ({r['pairs']} pairs in "
                              f"{r['seconds']:.1f} s); EGO reorder/sort untimed as in main.cu's egoTime"}
    import oracle
    n = db.shape[0]
    probe = np.linspace(0, n - 1, 64).astype(np.int64)
    _, t_probe = oracle.join_sample(db, wl.k, wl.eps, probe)
    m = int(max(64, min(n, 64 * seconds_target / max(t_probe, 1e-3))))
    qids = np.linspace(0, n - 1, m).astype(np.int64)
    pairs, sec = oracle.join_sample(db, wl.k, wl.eps, qids)
    return {"value": pairs / sec, "unit": "pairs/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{m} evenly spaced query points of the full {wl.name} dataset ({pairs} pairs in {sec:.1f} s); "
                      f"refine only, the index is built untimed"}


def load_workloads():
    """hegjoin_b200/workloads.py loaded by path: the workload table and the host
    generator (libhj_datagen.so) without importing the package, so the
    reference arm never loads the GPU library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("hj_workloads", os.path.join(ROOT, "hegjoin_b200", "workloads.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod      # dataclasses look their module up while the class is built
    spec.loader.exec_module(mod)
    return mod


L2_BYTES = 126 * 1000 * 1000


def dataset_bytes(wl) -> int:
    return wl.n * wl.d * (4 if wl.dtype == "f32" else 8)


def workload_config(wl):
    """The `config` both arms print for a workload (identical keys and values)."""
    mb = dataset_bytes(wl) / 1e6
    l2 = (f"inputs larger than L2 ({mb:.0f} MB dataset > 126 MB L2); no flush" if dataset_bytes(wl) > L2_BYTES else
          f"dataset ({mb:.0f} MB) fits in L2: a 512 MB buffer is written between timed steps (untimed)")
    return {"workload": wl.name, "n": wl.n, "d": wl.d, "k": wl.k, "eps": wl.eps, "dtype": wl.dtype,
            "seed": wl.seed, "l2": l2}


class HostRing:
    """A batch sink that reads every result pair on the host: each batch's neighbour
    ids are copied, in chunks, into a ring of two pinned host buffers on a copy stream
    of its own, which first waits for the batch on the join's stream.  The join runs
    with stream_overlap and reuses a batch's arrays only after the event this sink
    returns, so the copy of one batch overlaps the refine and grouping of the next."""

    def __init__(self, chunk_elems: int = 1 << 28):
        import torch
        self.torch = torch
        self.bufs = [torch.empty(chunk_elems, dtype=torch.int32).pin_memory() for _ in range(2)]
        self.copy = torch.cuda.Stream()
        self.events = []            # kept alive until the join returns
        self.chunk = chunk_elems
        self.bytes = 0
        self.i = 0

    def reset(self):
        self.events = []
        self.bytes = 0

    def __call__(self, batch, count, keys, vals, stream):
        import hegjoin_b200 as hj
        torch = self.torch
        join_stream = torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream()
        ready = torch.cuda.Event()
        ready.record(join_stream)
        self.copy.wait_event(ready)
        src = hj.device_view(vals, (count,), np.int32)
        with torch.cuda.stream(self.copy):
            # the ring's buffers are reused in copy-stream order: no host wait
            for off in range(0, count, self.chunk):
                m = min(self.chunk, count - off)
                self.bufs[self.i % 2][:m].copy_(src[off:off + m], non_blocking=True)
                self.i += 1
        done = torch.cuda.Event()
        done.record(self.copy)
        self.events.append((ready, done))
        self.bytes += 4 * count
        return 0, done.cuda_event


def reference_arm(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    db = wl.generate()
    # each step a bounded sample, so the whole run stays within a few minutes
    per_step = max(3.0, min(args.ref_seconds, 150.0 / max(1, args.steps + args.warmup)))
    steps = []
    base = None
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(db, wl, seconds_target=per_step)
        if i >= args.warmup:
            steps.append(b)
        base = b
    val = statistics.mean(s["value"] for s in steps)
    line = {"impl": "reference", "metric": "result pairs/s", "value": val, "unit": "pairs/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": wl.dtype, "data": "synthetic (seeded Exp(40) generator)",
            "config": workload_config(wl),
            "run": {"sample_per_step": base["sample"], "seconds_per_step_target": per_step},
            "cpu_baseline": {**base, "value": val},
            "e2e": {"value": val, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# serving (the request-stream workload): --serve
def quick_eps(db: np.ndarray, target: float, dev, seed: int) -> float:
    """Epsilon for a mean of `target` neighbours at the dataset's full size, from a pooled
    sample of query-to-point squared distances (256 queries x up to 100k points)."""
    import torch
    n = db.shape[0]
    rng = np.random.default_rng(seed)
    s = min(n, 100_000)
    ref = db if s == n else db[np.sort(rng.choice(n, s, replace=False))]
    q = db[rng.choice(n, min(256, n), replace=False)]
    R = torch.from_numpy(ref).to(dev)
    Q = torch.from_numpy(q).to(dev)
    d2 = torch.cdist(Q, R).square_().reshape(-1)
    level = min(1.0, target / n)
    r2 = torch.quantile(d2[torch.randperm(d2.numel(), device=dev)[:16_000_000]], level).item()
    return float(np.float32(np.sqrt(max(r2, 1e-12))))


def serving_run(n_requests: int, max_n: int, min_n: int = 1000, workers: int = 8, load: float = 5.0,
                hbm_budget_gb: float = 150.0, seed: int = 5, refine: str = "auto", with_plain: bool = True):
    """A seeded request stream through the serving loop: n log-uniform in [min_n, max_n],
    d from {2, 6, 18, 32, 90} (k = min(d, 6)), eps per request for a mean neighbour count
    drawn from U[4, 128].  Measures, on the same requests:
      serial        the same engine, one request at a time (all queued at t = 0, 1 worker);
      serial_plain  plain FP32 joins (exact refine), one at a time;
      capacity      all requests queued at once, `workers` in flight;
      served        Poisson arrivals at `load` x the serial same-engine request rate.
    Latency is per request, from submit to completion."""
    import threading
    import torch
    import hegjoin_b200 as hj
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n_requests):
        n = int(np.exp(rng.uniform(np.log(min_n), np.log(max_n))))
        d = int(rng.choice([2, 6, 18, 32, 90]))
        target = float(rng.uniform(4, 128))
        db = hj.generate_exp40(10_000 + i, n, d, np.float32)
        reqs.append((db, min(d, 6), quick_eps(db, target, dev, i), target))
    total_pts = sum(r[0].shape[0] for r in reqs)

    # one server per (workers, refine), created and warmed before any timed run: the
    # measurements are of a running service, not of its start-up (worker threads,
    # streams, workspaces)
    servers = {}

    def server(nworkers, refine_kind):
        key = (nworkers, refine_kind)
        if key not in servers:
            servers[key] = hj.Server(workers=nworkers, hbm_budget=int(hbm_budget_gb * (1 << 30)), refine=refine_kind)
        return servers[key]

    def run(nworkers, arrivals, todo=None, refine_kind=None):
        todo = reqs[:len(arrivals)] if todo is None else todo
        srv = server(nworkers, refine_kind or refine)
        tickets = [None] * len(todo)
        t0 = time.perf_counter()

        def submitter():
            for i, (db, k, eps, _) in enumerate(todo):
                delay = t0 + arrivals[i] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                tickets[i] = srv.submit(db, k, eps)

        th = threading.Thread(target=submitter)
        th.start()
        lat, pairs, infos = [], 0, []
        for i in range(len(todo)):
            while tickets[i] is None:
                time.sleep(0.0002)
            _, info = srv.wait(tickets[i], keep_result=False)
            lat.append(info.t_done - info.t_submit)
            pairs += info.stats.total_pairs
            infos.append(info)
        th.join()
        span = max(x.t_done for x in infos) - min(x.t_submit for x in infos)
        return {"pairs": int(pairs), "seconds": span, "pairs_per_s": pairs / span,
                "requests_per_s": len(todo) / span,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(np.mean(lat) * 1e3)}

    # warm-up of every server used below: one request of every dimension class per worker
    # (tile-shape tuning, memory pools, each worker's first allocations)
    first = {}
    for r in reqs:
        first.setdefault(r[0].shape[1], r)
    warm = list(first.values())
    run(1, np.zeros(len(warm)), warm)
    run(1, np.zeros(len(warm)), warm, refine_kind="exact")
    run(workers, np.zeros(len(warm) * workers), warm * workers)
    serial = run(1, np.zeros(len(reqs)))
    serial_plain = run(1, np.zeros(len(reqs)), refine_kind="exact") if with_plain else None
    capacity = run(workers, np.zeros(len(reqs)))
    rate = load * len(reqs) / serial["seconds"]
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    served = run(workers, arrivals)
    served["offered_seconds"] = float(arrivals[-1])
    for srv in servers.values():
        srv.close()
    out = {"requests": len(reqs), "points_total": int(total_pts), "n_range": [min_n, max_n],
           "d_choices": [2, 6, 18, 32, 90], "k": "min(d, 6)", "target_neighbours": "U[4, 128]",
           "arrivals": "Poisson", "offered_rate_req_per_s": rate,
           "offered_load": f"{load} x the serial same-engine request rate", "workers": workers,
           "hbm_budget_gb": hbm_budget_gb, "refine": refine,
           "served": served, "capacity": capacity, "serial": serial,
           "capacity_vs_serial": capacity["pairs_per_s"] / serial["pairs_per_s"],
           "served_vs_serial": served["pairs_per_s"] / serial["pairs_per_s"],
           "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"]}
    if serial_plain:
        out["serial_plain"] = serial_plain
        out["capacity_vs_serial_plain"] = capacity["pairs_per_s"] / serial_plain["pairs_per_s"]
        out["served_vs_serial_plain"] = served["pairs_per_s"] / serial_plain["pairs_per_s"]
    return out


def serve_bench(args):
    with ClockSampler(0) as clk:
        r = serving_run(args.requests, args.max_n, args.min_n, args.workers, args.load, args.hbm_budget_gb,
                        args.serve_seed, args.refine)
    line = {"metric": "served p50/p99 latency (ms) and aggregate result pairs/s", "value": r["served"]["pairs_per_s"],
            "unit": "pairs/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic request stream (seeded Exp(40) datasets)", "config": {"workload": "serving"},
            **r, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# tensor-core filter vs plain FP32 refine on one workload: --compare
def tc_vs_plain(wl, steps: int, warmup: int, tc_kind: str = "auto"):
    """The exact refine (plain FP32 on the CUDA cores) against the tensor-core
    filter on one workload: whole steps (index, workload order, join) timed with
    CUDA events on the launching stream, pair sets compared through per-query
    digests, and the filter's squared-distance error against FP64 on sampled tiles."""
    import torch
    import hegjoin_b200 as hj
    dev = torch.device("cuda", 0)
    np_db = wl.generate()
    db = torch.from_numpy(np_db).to(dev)
    stream = torch.cuda.current_stream(dev)
    out, digests = {}, {}
    for refine in ("exact", tc_kind):
        ms = []
        for it in range(warmup + steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            ix = hj.GridIndex(db, wl.k, wl.eps)
            cand = ix.sort_by_workload()
            res = hj.join(ix, refine=refine)
            e1.record(stream)
            torch.cuda.synchronize()
            if it >= warmup:
                ms.append(e0.elapsed_time(e1))
            st = res.stats
            if it == warmup + steps - 1:
                c, s_, x = res.digest()
                digests[refine] = (c.cpu().numpy(), s_.cpu().numpy(), x.cpu().numpy())
            res.close()
            ix.close()
        sec = statistics.mean(ms) / 1e3
        out[refine] = {"pairs": int(st.total_pairs), "seconds_per_step": sec, "pairs_per_s": st.total_pairs / sec,
                       "refine_used": {1: "exact", 2: "tc_f16", 3: "tc_bf16"}.get(int(st.refine_used)),
                       "refine_kernel_ms": st.ms_refine_kernel,
                       "join_ms": {"setup": st.ms_setup, "estimate": st.ms_estimate, "refine": st.ms_refine,
                                   "group": st.ms_group, "total": st.ms_total},
                       "batches": int(st.n_batches), "retries": int(st.n_retries), "band_pairs": int(st.band_pairs),
                       "tc_accepts": int(st.tc_accepts), "filter_delta": st.filter_delta,
                       "candidates": int(cand)}
    same = all(np.array_equal(a, b) for a, b in zip(digests["exact"], digests[tc_kind]))
    # max |D - d2_fp64| of the tensor-core squared distance over sampled tiles
    probe_kind = out[tc_kind]["refine_used"] if out[tc_kind]["refine_used"] != "exact" else "tc_f16"
    ix = hj.GridIndex(db, wl.k, wl.eps)
    ix.sort_by_workload()
    n = np_db.shape[0]
    torch.cuda.synchronize()
    P = hj.device_view(ix.views()[0], (n, wl.d), np.float32).double().cpu().numpy()   # points in cell order
    rng = np.random.default_rng(3)
    max_err, max_near = 0.0, 0.0
    for _ in range(16):
        a0 = int(rng.integers(0, max(1, n - 128)))
        b0 = int(rng.integers(0, max(1, n - 512)))
        acc, _, _ = hj.probe_tc_tile(ix, probe_kind, a0, b0)
        nc, nq = min(128, n - a0), min(512, n - b0)
        C = P[a0:a0 + nc]
        Q = P[b0:b0 + nq]
        d2 = ((C[:, None, :] - Q[None, :, :]) ** 2).sum(-1)
        err = np.abs(acc[:nc, :nq] - d2)
        near = d2 <= 4 * wl.eps * wl.eps
        max_err = max(max_err, float(err.max()))
        if near.any():
            max_near = max(max_near, float(err[near].max()))
    ix.close()
    del db
    torch.cuda.empty_cache()
    return {"workload": wl.name, "n": wl.n, "d": wl.d, "k": wl.k, "eps": wl.eps, "steps": steps, "warmup": warmup,
            "timing": "whole steps (index + workload order + join), CUDA events on the launching stream",
            "plain_fp32": out["exact"], "tc_filter": out[tc_kind],
            "speedup": out[tc_kind]["pairs_per_s"] / out["exact"]["pairs_per_s"],
            "identical_pair_sets": bool(same),
            "band_pairs": out[tc_kind]["band_pairs"], "filter_delta": out[tc_kind]["filter_delta"],
            "max_abs_d2_error_vs_fp64": max_err, "max_abs_d2_error_vs_fp64_within_2eps": max_near,
            "error_sample": f"16 random tiles of 128 candidates x 512 queries ({probe_kind} tile probe) "
                            f"against FP64 distances"}


def compare_bench(args, wl):
    with ClockSampler(0) as clk:
        r = tc_vs_plain(wl, args.steps, args.warmup, args.tc_kind)
    print(json.dumps({"metric": "result pairs/s, tensor-core filter vs plain FP32", **r, "clocks": clk.summary()}),
          flush=True)


# ---------------------------------------------------------------------------------------------
# the grid-index build and workload order alone: --index
def index_bench(args, wl):
    """GridIndex (cell ids, radix sort, cell table, gathered points, cell hash) plus
    sort_by_workload, timed with CUDA events, against their algorithmic bytes:
    build n*d*s read + n*d*s written in cell order + 12*n (u64 key + u32 id) +
    16*nC; workload order nC*(3^(k-1)*4 + 8) (one row lookup per stencil row)."""
    import torch
    import hegjoin_b200 as hj
    dev = torch.device("cuda", 0)
    np_db = wl.generate()
    db = torch.from_numpy(np_db).to(dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(512 * 1000 * 1000 // 4, dtype=torch.float32, device=dev)
    s = 4 if wl.dtype == "f32" else 8
    t_build, t_sort = [], []
    nc = 0
    for it in range(args.warmup + args.steps):
        flush.fill_(1.0)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        ix = hj.GridIndex(db, wl.k, wl.eps)
        e[1].record(stream)
        ix.sort_by_workload()
        e[2].record(stream)
        torch.cuda.synchronize()
        nc = ix.info().n_nonempty_cells
        ix.close()
        if it >= args.warmup:
            t_build.append(e[0].elapsed_time(e[1]))
            t_sort.append(e[1].elapsed_time(e[2]))
    pk, pk_kind = peaks()
    b_build = 2.0 * wl.n * wl.d * s + 12.0 * wl.n + 16.0 * nc
    b_sort = nc * (3 ** (wl.k - 1) * 4.0 + 8.0)
    mb, ms_ = statistics.mean(t_build), statistics.mean(t_sort)
    print(json.dumps({"metric": "grid-index build and workload order (achieved HBM GB/s)", "workload": wl.name,
                      "n": wl.n, "d": wl.d, "k": wl.k, "non_empty_cells": nc, "steps": args.steps,
                      "timing": "CUDA events on the launching stream; a 512 MB buffer written before each step",
                      "build": {"ms": mb, "algorithmic_bytes": b_build, "achieved_gbs": b_build / mb / 1e6,
                                "frac": b_build / mb / 1e6 / pk["hbm_gbs"]},
                      "workload_order": {"ms": ms_, "algorithmic_bytes": b_sort, "achieved_gbs": b_sort / ms_ / 1e6,
                                         "frac": b_sort / ms_ / 1e6 / pk["hbm_gbs"]},
                      "peak": {"hbm_gbs": pk["hbm_gbs"], "kind": f"{pk_kind} copy bandwidth"}}), flush=True)


# ---------------------------------------------------------------------------------------------
# dataset ingest at the skewed 6-D configuration's size: --ingest
def ingest_bench(args, wl):
    """The reference's text importer (import_dataset.cpp:10-40, restated in the oracle
    with the same stringstream calls, one thread) against hj_import_text (all host
    threads) and the binary twin, on the workload written in the reference
    generator's layout with max_digits10 significant digits."""
    import tempfile
    import hegjoin_b200 as hj
    import oracle
    db = wl.generate()
    digits = 9 if db.dtype == np.float32 else 17
    with tempfile.TemporaryDirectory() as tmp:
        txt, binp = os.path.join(tmp, "db.txt"), os.path.join(tmp, "db.hjds")
        oracle.write_text(txt, db, digits)
        size = os.path.getsize(txt)
        times = []
        for _ in range(2):
            t0 = time.perf_counter()
            got = hj.import_text(txt, wl.d, db.dtype)
            times.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        ref = oracle.import_text(txt, db.dtype)
        t_ref = time.perf_counter() - t0
        same = bool(np.array_equal(got.reshape(-1).view(np.uint8), ref.view(np.uint8))) and np.array_equal(got, db)
        hj.write_binary(binp, db)
        t0 = time.perf_counter()
        gb = hj.import_binary(binp, wl.d, db.dtype)
        t_bin = time.perf_counter() - t0
    print(json.dumps({"metric": "dataset ingest (values/s)", "workload": wl.name, "n": wl.n, "d": wl.d,
                      "text_bytes": size, "values": int(db.size), "identical_values": same,
                      "binary_identical": bool(np.array_equal(gb, db)),
                      "reference_stringstream": {"seconds": t_ref, "values_per_s": db.size / t_ref, "threads": 1},
                      "hj_import_text": {"seconds": min(times), "values_per_s": db.size / min(times),
                                         "threads": os.cpu_count()},
                      "hj_import_binary": {"seconds": t_bin, "values_per_s": db.size / t_bin},
                      "speedup_text": t_ref / min(times)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2_18d")
    ap.add_argument("--refine", default="auto")
    ap.add_argument("--n", type=int, default=0, help="override the workload's point count (testing only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--stream", action="store_true",
                    help="consume each batch instead of keeping the result (default for c1_2d)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the tensor-core-vs-plain (90-D) and serving blocks of the default line")
    ap.add_argument("--extra-steps", type=int, default=2)
    ap.add_argument("--ref-seconds", type=float, default=20.0)
    ap.add_argument("--serve", action="store_true", help="run the request-stream serving benchmark instead")
    ap.add_argument("--requests", type=int, default=256)
    ap.add_argument("--min-n", type=int, default=1000)
    ap.add_argument("--max-n", type=int, default=1_000_000)
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--load", type=float, default=5.0,
                    help="serving: Poisson arrival rate as a multiple of the serial same-engine request rate")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-seed", type=int, default=5)
    ap.add_argument("--compare", action="store_true", help="time the exact refine against the tensor-core filter")
    ap.add_argument("--tc-kind", default="auto", choices=["auto", "tc_f16", "tc_bf16"])
    ap.add_argument("--ingest", action="store_true", help="time the text importer against the reference's")
    ap.add_argument("--index", action="store_true", help="time the index build and workload order alone")
    ap.add_argument("--peaks", action="store_true", help="measure this library's pipe peaks (hj_measure_peaks)")
    args = ap.parse_args()
    if args.serve:
        serve_bench(args)
        return

    wlmod = load_workloads()
    wl = wlmod.WORKLOADS[args.workload]
    if args.n:
        import dataclasses
        wl = dataclasses.replace(wl, n=args.n)
    if args.impl == "reference":
        reference_arm(args, wl)
        return
    if args.compare:
        compare_bench(args, wl)
        return
    if args.ingest:
        ingest_bench(args, wl)
        return
    if args.index:
        index_bench(args, wl)
        return
    if args.peaks:
        import hegjoin_b200 as hj
        with ClockSampler(0) as clk:
            pk = hj.measure_peaks()
        print(json.dumps({"metric": "measured pipe peaks (TFLOP/s)", **pk, "clocks": clk.summary()}), flush=True)
        return

    import torch
    import torch.distributed as dist
    import hegjoin_b200 as hj
    ws, rank, local = dist_init()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    np_db = wl.generate()
    db = torch.from_numpy(np_db).to(dev)
    stream = torch.cuda.current_stream(dev)
    shard = dict(shard_count=ws, shard_index=rank) if ws > 1 else {}

    # results too large to keep on the device (the 2-D, 2M-point configuration: ~1.9e10
    # pairs, 76 GB of neighbour ids) go through the streamed join: each grouped batch is
    # consumed (per-query digests on the device) and its buffers reused
    stream_mode = args.stream or wl.name == "c1_2d"
    flush = torch.empty(512 * 1000 * 1000 // 4, dtype=torch.float32, device=dev) \
        if dataset_bytes(wl) <= L2_BYTES else None

    def one_step():
        ix = hj.GridIndex(db, wl.k, wl.eps)
        cand = ix.sort_by_workload()
        if stream_mode:
            st, _ = hj.join_stream(ix, None, digest=True, refine=args.refine, **shard)
            pairs = st.total_pairs
        else:
            res = hj.join(ix, refine=args.refine, **shard)
            st = res.stats
            pairs = res.total_pairs
            res.close()
        out = (pairs, cand, st.ms_refine_kernel, st.refine_launches, st.refine_used, st.band_pairs,
               st.tc_accepts, st.filter_delta, int(st.n_batches))
        ix.close()
        return out

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = hj.kernel_launch_count()
    recs = []
    ms = 0.0
    with ClockSampler(local) as clk:
        if flush is None:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                recs.append(one_step())
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
        else:
            # the dataset fits in L2: write a larger buffer before every step, outside the timing
            for _ in range(args.steps):
                flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                recs.append(one_step())
                e1.record(stream)
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
    barrier()
    torch.cuda.synchronize()
    launches = hj.kernel_launch_count() - launches0
    ms_step = ms / args.steps
    pairs = recs[-1][0]
    cand = recs[-1][1]
    kern_ms = statistics.mean(r[2] for r in recs)
    refine_used = recs[-1][4]
    band, acc, delta = recs[-1][5], recs[-1][6], recs[-1][7]
    # whole-job aggregates: pairs summed over ranks, time = max over ranks
    tot_pairs, = allreduce([float(pairs)], dist.ReduceOp.SUM) if ws > 1 else [float(pairs)]
    max_ms, max_kern = allreduce([ms_step, kern_ms], dist.ReduceOp.MAX) if ws > 1 else [ms_step, kern_ms]
    value = tot_pairs / (max_ms / 1e3)

    # roofline of the dominant kernel (the refine), algorithmic work per launch
    pk, pk_kind = peaks()
    tc = refine_used in (hj.HJ_REFINE_TC_F16, hj.HJ_REFINE_TC_BF16)
    cand_rank = cand / ws
    if tc:
        flops = 2.0 * wl.d * cand_rank
        peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
        achieved = flops / (kern_ms / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None, "kernel": "k_refine_tc",
                "peak_kind": f"{pk_kind} bf16 dense, sustained (kernel runs inside a seconds-long step)",
                "algorithmic": "2*d flops per candidate pair (C = sum over queries of stencil candidates)"}
    else:
        # queries read once, each 64-query block reads its candidates once, pairs written as two u32
        s = 4 if wl.dtype == "f32" else 8
        byts = (wl.n / ws) * wl.d * s + (cand_rank / 64.0) * wl.d * s + 8.0 * pairs
        achieved = byts / (kern_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / pk["hbm_gbs"], "traffic": None, "kernel": "k_refine_plain",
                "peak_kind": f"{pk_kind} copy bandwidth",
                "algorithmic": "n*d*s + (C/64)*d*s + 8*P bytes per launch"}
    traffic_path = os.path.join(ROOT, "profiles", f"traffic_{wl.name}.txt")
    if os.path.exists(traffic_path):
        try:
            tr = json.load(open(traffic_path))
            key = "tc" if tc else "plain"
            if key in tr:
                roof["traffic"] = tr[key]["bytes_per_launch_scaled"]
                roof["traffic_note"] = tr[key]["note"]
        except Exception:
            pass

    # end to end through the host entry point: pinned H2D in, full result D2H out
    e2e = None
    if not args.no_e2e and stream_mode:
        # streamed: pinned H2D of the dataset, the join, and every batch's neighbour ids
        # plus the per-query counts copied back to pinned host memory
        host_db = torch.from_numpy(np_db).pin_memory()
        ring = HostRing()
        e2e_ms, d2h = [], 0
        cnt_h = torch.empty(np_db.shape[0], dtype=torch.int32).pin_memory()
        for it in range(1 + args.steps):
            if flush is not None:
                flush.fill_(1.0)
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            ring.reset()
            d_db = host_db.to(dev, non_blocking=True)
            ix = hj.GridIndex(d_db, wl.k, wl.eps)
            ix.sort_by_workload()
            st, (c, _, _) = hj.join_stream(ix, ring, digest=True, refine=args.refine, stream_overlap=True, **shard)
            cnt_h.copy_(c, non_blocking=True)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            ix.close()
            del d_db
            d2h = ring.bytes + cnt_h.numel() * 4
            if it >= 1:
                e2e_ms.append((t1 - t0) * 1e3)
        e_ms = statistics.mean(e2e_ms)
        e_ms_max, = allreduce([e_ms], dist.ReduceOp.MAX) if ws > 1 else [e_ms]
        e2e = {"value": tot_pairs / (e_ms_max / 1e3), "unit": "pairs/s",
               "h2d_bytes_per_step": int(np_db.nbytes), "d2h_bytes_per_step": int(d2h), "ms_per_step": e_ms_max,
               "path": "pinned H2D, GridIndex + join_stream (stream_overlap); each batch's neighbour ids "
                       "copied to pinned host memory on a copy stream, overlapping the next batches; the "
                       "per-query counts copied at the end"}
    elif not args.no_e2e:
        host_db = torch.from_numpy(np_db).pin_memory()
        n = np_db.shape[0]
        off_h = torch.empty(n + 1, dtype=torch.int64).pin_memory()
        vals_h = None
        e2e_ms = []
        d2h = 0
        for it in range(2 + args.steps):
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            o = hj.join_opts(refine=args.refine, **shard)
            stt = hj.JoinStats()
            h = ctypes.c_void_p()
            hj.check(hj.lib.hj_self_join_host(host_db.data_ptr(), n, wl.d, wl.k,
                                              hj.HJ_F32 if wl.dtype == "f32" else hj.HJ_F64, float(wl.eps),
                                              ctypes.byref(o), hj._stream_ptr(None), ctypes.byref(h),
                                              ctypes.byref(stt)))
            res = hj.JoinResult(h, stt, n, dev)
            off_d, vals_d = res.to_csr(sort_lists=False)
            if vals_h is None or vals_h.numel() < vals_d.numel():
                vals_h = torch.empty(max(1, vals_d.numel()), dtype=torch.int32).pin_memory()
            off_h.copy_(off_d, non_blocking=True)
            vals_h[:vals_d.numel()].copy_(vals_d, non_blocking=True)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            d2h = off_d.numel() * 8 + vals_d.numel() * 4
            res.close()
            del off_d, vals_d
            if it >= 2:
                e2e_ms.append((t1 - t0) * 1e3)
        e_ms = statistics.mean(e2e_ms)
        e_ms_max, = allreduce([e_ms], dist.ReduceOp.MAX) if ws > 1 else [e_ms]
        e2e = {"value": tot_pairs / (e_ms_max / 1e3), "unit": "pairs/s",
               "h2d_bytes_per_step": int(np_db.nbytes), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e_ms_max}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(np_db, wl, seconds_target=20.0)

    # this library's own measured pipe peaks: a second denominator beside the driver's
    own = None
    if ws == 1 and not args.no_extras:
        own = hj.measure_peaks()
        if tc:
            roof["own_mma_peak_tflops"] = own["f16_mma_tflops"]
            roof["frac_of_own_mma_peak"] = roof["achieved"] / own["f16_mma_tflops"]

    # the north-star comparisons, each with its own clock record (single GPU only)
    extras = {}
    if ws == 1 and not args.no_extras and wl.name == "c2_18d":
        del db
        torch.cuda.empty_cache()
        with ClockSampler(local) as clk3:
            extras["tc_vs_plain"] = tc_vs_plain(wlmod.WORKLOADS["c3_90d"], args.extra_steps, 1)
        extras["tc_vs_plain"]["clocks"] = clk3.summary()
        t3 = extras["tc_vs_plain"]
        c3 = wlmod.WORKLOADS["c3_90d"]
        cand3 = t3["plain_fp32"]["candidates"]
        # plain FP32: 3 d flops per candidate (sub, multiply, add) on the FP32 pipe; the filter:
        # 2 d per candidate on the tensor pipe (the MMA itself does 2 Kpad)
        for arm, flops_per, peak_key in (("plain_fp32", 3.0 * c3.d, "fp32x2_fma_tflops"),
                                          ("tc_filter", 2.0 * c3.d, "f16_mma_tflops")):
            ach = flops_per * cand3 / (t3[arm]["refine_kernel_ms"] / 1e3) / 1e12
            t3[arm]["roofline"] = {"achieved_tflops": ach, "own_peak_tflops": own[peak_key],
                                   "frac_of_own_peak": ach / own[peak_key], "peak": peak_key}
        with ClockSampler(local) as clk5:
            extras["serving"] = serving_run(96, 100_000, workers=8, load=5.0, seed=args.serve_seed)
        extras["serving"]["clocks"] = clk5.summary()
        extras["serving"]["stream"] = ("96 requests, n log-uniform in [1e3, 1e5] (the full request stream of "
                                       "4,096 requests up to 1e6 points runs with --serve)")
        with ClockSampler(local) as clk6:
            extras["serving_small"] = serving_run(256, 20_000, workers=8, load=5.0, seed=args.serve_seed + 1)
        extras["serving_small"]["clocks"] = clk6.summary()
        extras["serving_small"]["stream"] = "256 small requests, n log-uniform in [1e3, 2e4]"

    if rank == 0:
        line = {
            "metric": "result pairs/s", "value": value, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": wl.dtype,
            "data": "synthetic (seeded Exp(40) generator, counter-based; no dataset is shipped)",
            "config": workload_config(wl),
            "run": {"refine": {1: "exact", 2: "tc_f16", 3: "tc_bf16"}.get(refine_used, str(refine_used)),
                    "pairs_per_step": int(tot_pairs), "candidates_per_step": int(cand),
                    "band_pairs": int(band), "tc_accepts": int(acc), "filter_delta": delta,
                    "refine_kernel_ms": max_kern, "batches": int(recs[-1][8]),
                    "result": "streamed: per-query digests on the device, batches not kept" if stream_mode else
                              "kept on the device (per-batch neighbour ids + neighbour table)",
                    "parallelism": f"query-block shards x{ws}" if ws > 1 else "single GPU"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk.summary(), "peaks_own": own, **extras,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
