"""Golden per-query neighbour counts of the 2-D FP64 configuration at full size.

Runs the CPU oracle's count-only join (oracle/hj_oracle.cpp) on the seeded
2,000,000-point dataset of hegjoin_b200.workloads ("c1_2d": seed 0,
eps = 0.002, k = 2) and stores the total pair count and a SHA-256 of the
2,000,000 counts (uint32, little-endian, by original query id).  The count
pass takes a few minutes of CPU, so the GPU test compares against this file
instead of re-running it.

    python tests/golden/make_c1_counts.py
"""
import hashlib
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import oracle  # noqa: E402
from hegjoin_b200 import workloads  # noqa: E402


def main():
    wl = workloads.WORKLOADS["c1_2d"]
    db = wl.generate()
    t0 = time.time()
    mn, _, nc, _ = oracle.geometry(db, wl.k, wl.eps)
    off, _ = oracle.join(db, wl.k, wl.eps, mn, nc, lists=False)
    counts = np.diff(off).astype("<u4")
    out = {"workload": wl.name, "n": wl.n, "d": wl.d, "k": wl.k, "eps": wl.eps, "seed": wl.seed,
           "total_pairs": int(off[-1]), "counts_sha256": hashlib.sha256(counts.tobytes()).hexdigest(),
           "max_count": int(counts.max()), "oracle_seconds": round(time.time() - t0, 1)}
    with open(os.path.join(ROOT, "tests", "golden", "c1_2d_counts.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
