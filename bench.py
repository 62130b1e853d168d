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


def cpu_baseline(db, wl, seconds_target=20.0):
    """The CPU restatement of the refine on a bounded query sample, all host threads."""
    import oracle
    n = db.shape[0]
    # calibrate the sample size on 64 queries, then size it for ~seconds_target
    probe = np.linspace(0, n - 1, 64).astype(np.int64)
    _, t_probe = oracle.join_sample(db, wl.k, wl.eps, probe)
    m = int(max(64, min(n, 64 * seconds_target / max(t_probe, 1e-3))))
    qids = np.linspace(0, n - 1, m).astype(np.int64)
    pairs, sec = oracle.join_sample(db, wl.k, wl.eps, qids)
    return {"value": pairs / sec, "unit": "pairs/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{m} evenly spaced query points of the full {wl.name} dataset ({pairs} pairs in {sec:.1f} s); "
                      f"refine only, the index is built untimed"}


def reference_arm(args, wl):
    ws, rank, local = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    db = wl.generate()
    steps = []
    base = None
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(db, wl, seconds_target=args.ref_seconds)
        if i >= args.warmup:
            steps.append(b)
        base = b
    val = statistics.mean(s["value"] for s in steps)
    line = {"impl": "reference", "metric": "result pairs/s", "value": val, "unit": "pairs/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": wl.dtype, "data": "synthetic (seeded Exp(40) generator)",
            "config": {"workload": wl.name, "n": wl.n, "d": wl.d, "k": wl.k, "eps": wl.eps},
            "cpu_baseline": {**base, "value": val},
            "e2e": {"value": val, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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
    ap.add_argument("--ref-seconds", type=float, default=20.0)
    args = ap.parse_args()

    from hegjoin_b200 import workloads
    wl = workloads.WORKLOADS[args.workload]
    if args.n:
        import dataclasses
        wl = dataclasses.replace(wl, n=args.n)
    if args.impl == "reference":
        reference_arm(args, wl)
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

    def one_step():
        ix = hj.GridIndex(db, wl.k, wl.eps)
        cand = ix.sort_by_workload()
        res = hj.join(ix, refine=args.refine, **shard)
        st = res.stats
        out = (res.total_pairs, cand, st.ms_refine_kernel, st.refine_launches, st.refine_used, st.band_pairs,
               st.tc_accepts, st.filter_delta)
        res.close()
        ix.close()
        return out

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = hj.kernel_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    recs = []
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            recs.append(one_step())
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches = hj.kernel_launch_count() - launches0
    ms = e0.elapsed_time(e1)
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
    traffic_path = os.path.join(ROOT, "profiles", f"traffic_{wl.name}.json")
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
    if not args.no_e2e:
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

    if rank == 0:
        line = {
            "metric": "result pairs/s", "value": value, "unit": "pairs/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": wl.dtype,
            "data": "synthetic (seeded Exp(40) generator, counter-based; no dataset is shipped)",
            "config": {"workload": wl.name, "n": wl.n, "d": wl.d, "k": wl.k, "eps": wl.eps,
                       "refine": {1: "exact", 2: "tc_f16", 3: "tc_bf16"}.get(refine_used, str(refine_used)),
                       "pairs_per_step": int(tot_pairs), "candidates_per_step": int(cand),
                       "band_pairs": int(band), "tc_accepts": int(acc), "filter_delta": delta,
                       "refine_kernel_ms": max_kern,
                       "l2": "inputs larger than L2 (dataset 360 MB > 126 MB); no flush",
                       "parallelism": f"query-block shards x{ws}" if ws > 1 else "single GPU"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
