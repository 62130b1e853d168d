"""Times the reference's own GPU-only join (algorithm 0) beside this library's, on
one of the benchmark workloads -- test infrastructure, not part of the library.

The reference is the lookup-fixed build of its own sources (oracle/ref/Makefile,
CFG=r90d for the 90-D workload, r18d for 18-D), driven by ref_driver, which
replays main.cu's algorithm-0 sequence and prints its phase times (s_index,
s_sort, s_join).  The reference writes its result buffers without a bounds check
(kernel.cu:357-359), so before it runs, its batch plan (GPUBatchEst_v2,
GPU.cu:403-779) is replayed on the CPU from the exact per-query counts and the
reference's own std::sort cell order; it runs only if no batch can reach its
buffer.  The per-query counts come from this library, whose counts equal the
oracle's at every benchmark configuration's full size (tests/test_gpu_parity_full.py).

    python oracle/ref/time_reference_gpu.py --workload c3_90d --out gpurun_out/ref_c3.json
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

BUILD_FOR = {18: "r18d", 90: "r90d"}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c3_90d")
    ap.add_argument("--n", type=int, default=0, help="point count (default: the workload's)")
    ap.add_argument("--timeout", type=float, default=600.0)
    ap.add_argument("--out", default="")
    a = ap.parse_args()

    import torch

    import hegjoin_b200 as hj
    import oracle
    from hegjoin_b200 import workloads

    wl = workloads.WORKLOADS[a.workload]
    db = wl.generate(a.n) if a.n else wl.generate()
    n, d = db.shape
    build = BUILD_FOR.get(d)
    exe = os.path.join(ROOT, "oracle", "_ref", build or "none", "ref_driver")
    if build is None or not os.path.exists(exe) or wl.k != 6 or db.dtype != np.float32:
        print(json.dumps({"unavailable": f"no reference build for d={d}, k={wl.k}, {db.dtype}"}))
        return 0

    # this library, timed whole (index + workload order + join), and its per-query counts
    dev = torch.device("cuda:0")
    x = torch.from_numpy(db).to(dev)
    times = []
    for rep in range(3):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        ix = hj.GridIndex(x, wl.k, wl.eps)
        ix.sort_by_workload()
        res = hj.join(ix)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
        if rep < 2:
            res.close()
            del ix
    counts = res.digest()[0].cpu().numpy().astype(np.int64)
    ours_pairs = int(res.total_pairs)
    refine_used = int(res.stats.refine_used)
    res.close()

    # the reference's batch plan, replayed on the CPU
    mn, _, nc, _ = oracle.geometry(db, wl.k, wl.eps)
    lid, first, last, lookup = oracle.index(db, wl.k, wl.eps, mn, nc)
    nb, _ = oracle.cell_workload(db, wl.k, wl.eps, mn, nc)
    order = oracle.ref_cell_order(nb)
    origin = np.concatenate([lookup[first[c]:last[c] + 1] for c in order])
    buf, batches, actual = oracle.ref_batches(counts, origin)
    safe = buf >= 100 and len(batches) >= 4 and max(actual) < 2 * buf
    rec = {"workload": a.workload, "n": int(n), "d": int(d), "k": wl.k, "eps": float(wl.eps),
           "ours": {"seconds_per_join": min(times), "pairs": ours_pairs, "refine_used": refine_used,
                    "timing": "index + workload order + join, CUDA events, best of 3"},
           "reference_plan": {"gpu_buffer_size": int(buf), "batches": len(batches),
                              "max_batch_pairs": int(max(actual)), "safe": bool(safe)}}
    if not safe:
        rec["reference"] = {"skipped": "its batch plan could overflow its unchecked result buffer"}
    else:
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "db.bin")
            with open(path, "wb") as f:
                np.array([n, d, db.dtype.itemsize], np.uint32).tofile(f)
                db.tofile(f)
            t0 = time.time()
            try:
                p = subprocess.run([exe, path, repr(float(wl.eps)), os.path.join(tmp, "out")], capture_output=True,
                                   text=True, timeout=a.timeout)
            except subprocess.TimeoutExpired:
                rec["reference"] = {"error": f"did not finish within {a.timeout} s"}
                p = None
            wall = time.time() - t0
            if p is not None:
                lines = [l for l in p.stdout.splitlines() if l.startswith("HJREF ")]
                if p.returncode != 0 or not lines:
                    rec["reference"] = {"error": f"rc={p.returncode}", "stderr": p.stderr[-1000:]}
                else:
                    meta = json.loads(lines[-1][6:])
                    meta["wall_seconds_incl_dumps"] = wall
                    meta["seconds_index_sort_join"] = meta["s_index"] + meta["s_sort"] + meta["s_join"]
                    meta["pairs_equal_ours"] = int(meta["total_neighbors"]) == ours_pairs
                    rec["reference"] = meta
                    rec["speedup_ours_vs_reference"] = meta["seconds_index_sort_join"] / min(times)
    print(json.dumps(rec), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(rec, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
