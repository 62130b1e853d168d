"""Golden fixtures from the reference itself.

Builds (here, where the reference sources are) and runs (on a GPU machine) the
reference's own GPU-only join through oracle/_ref/<cfg>/ref_driver -- the
reference's GPU.cu / SortByWorkload.cu / kernel.cu compiled by
oracle/ref/Makefile, with the one build fix that makes its cell-lookup
comparator callable on the device -- on seeded datasets from
hegjoin_b200.workloads, and stores what it computed as small .npz fixtures in
tests/golden/:

  geometry (minArr, nCells, totalCells), the index arrays (cell ids, grid
  first/last, indexLookupArr), the workload order (schedulingCell pairs,
  originPointIndex, totalCandidates), totalNeighbors, and per query the
  neighbour count and an order-independent digest of its neighbour ids.

The datasets themselves are not stored; they are regenerated from the spec.

Safety: before the reference runs, its batch plan (GPUBatchEst_v2) is replayed
on the CPU from the oracle's exact per-query counts and the reference's own
std::sort order.  A case whose largest batch could reach the reference's
result buffer (2 x GPUBufferSize pairs, GPU.cu:1042-1062, written without a
bounds check at kernel.cu:357-359) is skipped, never run.

    python tests/golden/make_ref_fixtures.py --build        # where the reference sources are (HJ_REFERENCE_DIR)
    python tests/golden/make_ref_fixtures.py --run OUTDIR   # on the GPU machine
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# build name -> (GPUNUMDIM, NUMINDEXEDDIM, DTYPE)
BUILDS = {
    "r2d": (2, 2, "double"),
    "r6d": (6, 6, "float"),
    "r18d": (18, 6, "float"),
    "r90d": (90, 6, "float"),
    "r5k3": (5, 3, "double"),
}

# fixture name, build, n, seed, eps, generator
CASES = [
    ("r2d_f64_dense", "r2d", 20000, 100, 0.01, "exp40"),
    ("r2d_f64_sparse", "r2d", 6000, 101, 0.004, "exp40"),
    ("r5k3_f64_exp", "r5k3", 8000, 106, 0.05, "exp40"),
    ("r2d_f64_edge", "r2d", 3000, 108, 0.02, "exp40"),
    ("r18d_f32_exp", "r18d", 8000, 102, 0.08, "exp40"),
    ("r90d_f32_exp", "r90d", 4000, 103, 0.25, "exp40"),
    ("r6d_f32_skewed", "r6d", 20000, 110, 0.02, "skewed"),
]
# An earlier run of a 6-D build (n=20000, eps 0.05) did not finish within 900 s.
# That build was compiled without the lookup fix (oracle/ref/Makefile), so every
# cell lookup resolved to the first non-empty cell and the candidate and result
# counts exploded.  The 6-D case above runs the lookup-fixed build, gated like
# every case by the batch-plan replay.
NOT_RUN = set()


def dataset(build, n, seed, gen):
    from hegjoin_b200 import workloads
    d, k, t = BUILDS[build]
    dt = np.float32 if t == "float" else np.float64
    if gen == "skewed":
        return workloads.skewed(seed, n, d, dtype=dt), k
    return workloads.exp40(seed, n, d, dt), k


def fold_digest(s, x):
    z = (s.astype(np.uint64) ^ ((x.astype(np.uint64) << np.uint64(1)) | (x.astype(np.uint64) >> np.uint64(63))))
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(31))) * np.uint64(0x9E3779B97F4A7C15)
    return z ^ (z >> np.uint64(29))


def build():
    for name, (d, k, t) in BUILDS.items():
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle", "ref"), "-j8", f"CFG={name}", f"D={d}",
                        f"K={k}", f"T={t}"], check=True, stdout=subprocess.DEVNULL)


def plan_is_safe(db, k, eps):
    """Replays the reference's batch plan; returns (safe, info)."""
    import oracle
    mn, _, nc, _ = oracle.geometry(db, k, eps)
    lid, first, last, lookup = oracle.index(db, k, eps, mn, nc)
    nb, _ = oracle.cell_workload(db, k, eps, mn, nc)
    order = oracle.ref_cell_order(nb)
    origin = np.concatenate([lookup[first[c]:last[c] + 1] for c in order])
    off, _ = oracle.join(db, k, eps, mn, nc, lists=False)
    counts = np.diff(off).astype(np.int64)
    buf, batches, actual = oracle.ref_batches(counts, origin)
    safe = buf >= 100 and len(batches) >= 4 and max(actual) < 2 * buf
    return safe, {"gpu_buffer_size": int(buf), "batches": len(batches), "max_batch_pairs": int(max(actual)),
                  "total_pairs": int(counts.sum())}


def run(outdir, only=None):
    import oracle
    os.makedirs(outdir, exist_ok=True)
    summary = {}
    for name, b, n, seed, eps, gen in CASES:
        if b in NOT_RUN or (only and name not in only):
            continue
        db, k = dataset(b, n, seed, gen)
        safe, info = plan_is_safe(db, k, eps)
        summary[name] = {"plan": info, "safe": bool(safe)}
        if not safe:
            print(f"{name}: skipped, the reference's batch plan could overflow its buffer: {info}", flush=True)
            continue
        exe = os.path.join(ROOT, "oracle", "_ref", b, "ref_driver")
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "db.bin")
            with open(path, "wb") as f:
                np.array([n, db.shape[1], db.dtype.itemsize], np.uint32).tofile(f)
                db.tofile(f)
            pre = os.path.join(tmp, "out")
            try:
                p = subprocess.run([exe, path, repr(float(eps)), pre], capture_output=True, text=True, timeout=240)
            except subprocess.TimeoutExpired:
                print(f"{name}: reference run exceeded 240 s; stopped, not retried", flush=True)
                summary[name]["error"] = "timeout"
                continue
            if p.returncode != 0:
                print(f"{name}: reference run failed rc={p.returncode}\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
                summary[name]["error"] = p.returncode
                continue
            line = [l for l in p.stdout.splitlines() if l.startswith("HJREF ")][-1]
            meta = json.loads(line[6:])
            d, kk, dt = db.shape[1], k, db.dtype
            g = open(pre + ".geom.bin", "rb").read()
            mn = np.frombuffer(g, dt, kk)
            nc = np.frombuffer(g, np.uint32, kk, kk * dt.itemsize)
            tot = np.frombuffer(g, np.uint64, 1, kk * dt.itemsize + 4 * kk)[0]
            ib = open(pre + ".index.bin", "rb").read()
            ncell = int(np.frombuffer(ib, np.uint32, 1)[0])
            o = 4
            lid = np.frombuffer(ib, np.uint64, ncell, o); o += 8 * ncell
            idx = np.frombuffer(ib, np.uint32, ncell, o); o += 4 * ncell
            gmin = np.frombuffer(ib, np.int32, ncell, o); o += 4 * ncell
            gmax = np.frombuffer(ib, np.int32, ncell, o); o += 4 * ncell
            ilu = np.frombuffer(ib, np.uint32, n, o)
            sb = open(pre + ".sched.bin", "rb").read()
            tcand = int(np.frombuffer(sb, np.uint64, 1)[0])
            sched = np.frombuffer(sb, np.int32, 2 * ncell, 8).reshape(ncell, 2)
            origin = np.frombuffer(sb, np.uint32, n, 8 + 8 * ncell)
            pb = open(pre + ".pairs.bin", "rb").read()
            tneigh, tsum = np.frombuffer(pb, np.uint64, 2)
            off = np.frombuffer(pb, np.uint64, n + 1, 16)
            vals = np.frombuffer(pb, np.uint32, int(tsum), 16 + 8 * (n + 1))
            cnt, s, x = oracle.digest(off, vals)
            np.savez_compressed(
                os.path.join(outdir, f"{name}.npz"),
                spec=np.array(json.dumps({"name": name, "build": b, "n": n, "d": d, "k": kk, "dtype": str(dt),
                                          "seed": seed, "eps": eps, "gen": gen})),
                min_arr=mn, n_cells=nc, total_cells=np.array(tot), cell_lid=lid, cell_idx=idx, grid_min=gmin,
                grid_max=gmax, index_lookup=ilu, total_candidates=np.array(tcand), sched=sched,
                origin_point_index=origin, total_neighbors=np.array(tneigh), table_pairs=np.array(tsum),
                counts=cnt.astype(np.uint32), digest=fold_digest(s, x))
            summary[name].update(meta)
            print(f"{name}: {json.dumps(meta)}", flush=True)
    with open(os.path.join(outdir, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--build", action="store_true")
    ap.add_argument("--run", metavar="OUTDIR")
    ap.add_argument("--only", nargs="*", help="run these cases only")
    a = ap.parse_args()
    if a.build:
        build()
    if a.run:
        run(a.run, a.only)
