"""Tensor-core filter: MMA plumbing against FP64 dot products, and the joined
pair set against the oracle (it must equal the exact path bit for bit)."""
import numpy as np
import pytest

import oracle
from hegjoin_b200 import workloads

pytestmark = pytest.mark.gpu


def _index(db, k, eps, dev):
    import torch
    import hegjoin_b200 as hj
    mn, _, nc, _ = oracle.geometry(db, k, eps)
    ix = hj.GridIndex(torch.from_numpy(db).to(dev), k, float(eps), [float(x) for x in mn], [int(x) for x in nc])
    return ix, mn, nc


@pytest.mark.parametrize("refine", ["tc_f16", "tc_bf16"])
@pytest.mark.parametrize("d", [18, 32, 90])
def test_tile_probe_matches_fp64(cuda, refine, d):
    import hegjoin_b200 as hj
    db = workloads.exp40(40, 3000, d, np.float32)
    ix, _, _ = _index(db, 6, 0.1, cuda)
    for a0, b0 in ((0, 0), (777, 1500), (2999, 2600)):
        acc, q, c = hj.probe_tc_tile(ix, refine, a0, b0)
        nq = min(512, 3000 - b0)
        nc = min(128, 3000 - a0)
        exp = c[:nc] @ q[:nq].T                      # candidate form . query form
        terms = np.abs(c[:nc]) @ np.abs(q[:nq]).T
        err = np.abs(acc[:nc, :nq] - exp)
        assert (err <= 1e-5 * terms + 1e-30).all(), float((err / (terms + 1e-30)).max())
        # rows beyond the dataset read zeros (TMA out-of-bounds fill)
        if nc < 128:
            assert np.all(acc[nc:, :nq] == 0)


CASES = [
    (4000, 18, 6, 0.06),
    (2500, 18, 6, 0.09),
    (1500, 90, 6, 0.25),
    (1200, 32, 6, 0.12),
    (3000, 16, 4, 0.08),
    (800, 64, 3, 0.2),
]


def _csr(res):
    off, vals = res.to_csr(sort_lists=True)
    return off.cpu().numpy().astype(np.uint64), vals.cpu().numpy().astype(np.uint32)


@pytest.mark.parametrize("refine", ["tc_f16", "tc_bf16"])
@pytest.mark.parametrize("n,d,k,eps", CASES)
def test_tc_join_equals_oracle(cuda, refine, n, d, k, eps):
    import hegjoin_b200 as hj
    db = workloads.exp40(41, n, d, np.float32)
    ix, mn, nc = _index(db, k, eps, cuda)
    res = hj.join(ix, refine=refine)
    off, vals = oracle.join(db, k, eps, mn, nc)
    goff, gvals = _csr(res)
    st = res.stats
    assert st.refine_used == hj.REFINE_NAMES[refine]
    assert res.total_pairs == int(off[-1])
    assert np.array_equal(goff, off)
    assert np.array_equal(gvals, vals)
    assert st.tc_accepts + st.band_pairs >= res.total_pairs


def test_tc_join_medium_digest_and_band(cuda):
    import hegjoin_b200 as hj
    db = workloads.exp40(42, 60000, 18, np.float32)
    k, eps = 6, 0.045
    ix, mn, nc = _index(db, k, eps, cuda)
    off, vals = oracle.join(db, k, eps, mn, nc)
    cnt, s, x = oracle.digest(off, vals)
    for refine in ("tc_f16", "tc_bf16"):
        res = hj.join(ix, refine=refine)
        gc, gs, gx = (t.cpu().numpy() for t in res.digest())
        assert np.array_equal(gc.astype(np.uint32), cnt)
        assert np.array_equal(gs.view(np.uint64), s)
        assert np.array_equal(gx.view(np.uint64), x)
        assert res.stats.band_pairs > 0 and res.stats.tc_accepts > 0


def test_tc_overflow_retry(cuda):
    import hegjoin_b200 as hj
    db = workloads.exp40(43, 20000, 18, np.float32)
    ix, mn, nc = _index(db, 6, 0.07, cuda)
    ref = hj.join(ix, refine="exact")
    small = hj.join(ix, refine="tc_f16", result_capacity=max(1, ref.total_pairs // 5))
    assert small.total_pairs == ref.total_pairs
    assert all(np.array_equal(a, b) for a, b in zip(_csr(small), _csr(ref)))
