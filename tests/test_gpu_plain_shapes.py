"""Both tile shapes of the exact refine give the reference's pair set.

The join times the two shapes (64 queries x 128 candidates and 64 x 64 per
staged chunk) on its estimator sample once per (d, dtype) and process and
keeps the faster, so each shape is forced in a child process of its own
through a tuning file (the library reads "kind d dtype shape" lines from
HJ_TUNE_FILE; kind 1 is the exact refine, dtype 0 float and 1 double).  The
cases cover the block path (k < 4, and large cells) and the warp path for
one-point cells (k >= 4), in float and double, with specialised and generic d.
"""
import json
import os
import subprocess
import sys
import textwrap

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import json, sys
    import numpy as np, torch
    sys.path.insert(0, {root!r})
    import oracle
    import hegjoin_b200 as hj
    from hegjoin_b200 import workloads
    out = []
    for n, d, k, eps, dt, gen in {cases!r}:
        dtype = np.float64 if dt == 1 else np.float32
        db = (workloads.skewed(44, n, d, dtype=dtype) if gen == "skewed"
              else workloads.exp40(44, n, d, dtype))
        ix = hj.GridIndex(torch.from_numpy(db).cuda(), k, eps)
        res = hj.join(ix, refine="exact")
        off, vals = res.to_csr(sort_lists=True)
        ref_off, ref_vals = oracle.join(db, k, eps)
        out.append(bool(np.array_equal(off.cpu().numpy().astype(np.uint64), ref_off)
                        and np.array_equal(vals.cpu().numpy().astype(np.uint32), ref_vals)))
    print("RESULT " + json.dumps(out))
""")

# n, d, k, eps, dtype (0 float, 1 double), generator
CASES = [(20000, 2, 2, 0.004, 1, "exp40"), (20000, 2, 2, 0.004, 0, "exp40"), (30000, 6, 6, 0.02, 0, "skewed"),
         (8000, 5, 5, 0.03, 1, "exp40"), (6000, 18, 6, 0.07, 0, "exp40")]


@pytest.mark.parametrize("shape", [0, 1])
def test_plain_shape_matches_oracle(cuda, tmp_path, shape):
    tune = tmp_path / "tune.txt"
    tune.write_text("".join(f"1 {d} {dt} {shape}\n" for _, d, _, _, dt, _ in CASES))
    env = dict(os.environ, HJ_TUNE_FILE=str(tune))
    code = CHILD.format(root=ROOT, cases=CASES)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    line = [l for l in p.stdout.splitlines() if l.startswith("RESULT ")][-1]
    assert all(json.loads(line[7:])), line
