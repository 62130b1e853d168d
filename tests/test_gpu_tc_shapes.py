"""Every epilogue shape of the tensor-core filter gives the exact pair set.

The autotuner picks one shape per (refine kind, d, dtype) and process, so each
shape is forced in a child process of its own through a tuning file (the
library reads "kind d dtype shape" lines from HJ_TUNE_FILE).  Shapes: 2 or 4
epilogue warp groups, shared by both accumulators (2, 4) or split into one set
per accumulator (10, 12); each with one vote per chunk or one per accumulator
(HJ_TC_DEFER=0/1; the library otherwise picks by the estimated pair density).
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
    for n, d, k, eps in {cases!r}:
        db = workloads.exp40(43, n, d, np.float32)
        ix = hj.GridIndex(torch.from_numpy(db).cuda(), k, eps)
        res = hj.join(ix, refine={refine!r})
        off, vals = res.to_csr(sort_lists=True)
        ref_off, ref_vals = oracle.join(db, k, eps)
        out.append(bool(np.array_equal(off.cpu().numpy().astype(np.uint64), ref_off)
                        and np.array_equal(vals.cpu().numpy().astype(np.uint32), ref_vals)))
    print("RESULT " + json.dumps(out))
""")

CASES = [(6000, 18, 6, 0.07), (2500, 90, 6, 0.26), (700, 32, 6, 0.2)]


@pytest.mark.parametrize("defer", ["0", "1"])
@pytest.mark.parametrize("refine,kind", [("tc_f16", 2), ("tc_bf16", 3)])
@pytest.mark.parametrize("shape", [2, 4, 10, 12])
def test_shape_matches_oracle(cuda, tmp_path, refine, kind, shape, defer):
    tune = tmp_path / "tune.txt"
    tune.write_text("".join(f"{kind} {d} 0 {shape}\n" for _, d, _, _ in CASES))
    env = dict(os.environ, HJ_TUNE_FILE=str(tune), HJ_TC_DEFER=defer)
    code = CHILD.format(root=ROOT, cases=CASES, refine=refine)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    line = [l for l in p.stdout.splitlines() if l.startswith("RESULT ")][-1]
    assert all(json.loads(line[7:])), line
