"""Tensor-core filter on data of any range, and at the threshold's edges.

The filter stores (x - min) * 2^s in FP16 or BF16, with s chosen per dataset,
so coordinates in raw units (thousands) or tiny ones (1e-3 scale) must give the
oracle's pair set bit for bit under every refine kind.  Pairs built to sit
exactly at the squared threshold T and one float either side, and pairs spread
through the guard band at the largest norms of the dataset, must also match.
"""
import numpy as np
import pytest

import oracle
from hegjoin_b200 import workloads

pytestmark = pytest.mark.gpu


def _index(db, k, eps, dev):
    import torch
    import hegjoin_b200 as hj
    mn, _, nc, _ = oracle.geometry(db, k, eps)
    ix = hj.GridIndex(torch.from_numpy(np.ascontiguousarray(db)).to(dev), k, float(eps),
                      [float(x) for x in mn], [int(x) for x in nc])
    return ix, mn, nc


def _csr(res):
    off, vals = res.to_csr(sort_lists=True)
    return off.cpu().numpy().astype(np.uint64), vals.cpu().numpy().astype(np.uint32)


def _check_all_kinds(db, k, eps, dev, kinds=("auto", "tc_f16", "tc_bf16", "exact")):
    import hegjoin_b200 as hj
    ix, mn, nc = _index(db, k, eps, dev)
    off, vals = oracle.join(db, k, eps, mn, nc)
    used = {}
    for refine in kinds:
        res = hj.join(ix, refine=refine)
        goff, gvals = _csr(res)
        assert res.total_pairs == int(off[-1]), refine
        assert np.array_equal(goff, off), refine
        assert np.array_equal(gvals, vals), refine
        used[refine] = int(res.stats.refine_used)
    return off, vals, used


@pytest.mark.parametrize("scale", [1000.0, 1e-3])
@pytest.mark.parametrize("d,k,eps,n", [(18, 6, 0.06, 3000), (90, 6, 0.25, 1500)])
def test_scaled_data_all_kinds_match_oracle(cuda, scale, d, k, eps, n):
    import hegjoin_b200 as hj
    db = (workloads.exp40(60, n, d, np.float32) * np.float32(scale)).astype(np.float32)
    e = np.float32(eps * scale)
    off, _, used = _check_all_kinds(db, k, e, cuda)
    assert off[-1] > n                               # more than the self pairs
    assert used["auto"] == hj.HJ_REFINE_TC_F16       # FP16 stays usable at any scale


def test_offset_far_from_zero(cuda):
    # coordinates around 3e3 with neighbours 0.1 apart: the origin shift removes the offset
    base = workloads.exp40(61, 2500, 18, np.float32)
    db = (base * np.float32(40.0) + np.float32(3000.0)).astype(np.float32)
    _check_all_kinds(db, 6, np.float32(2.4), cuda)


def _tie_dataset(d, eps, rng, n_base=120):
    """Base points and partners whose fma-chain squared distance is exactly T,
    the float below T and the float above T.  Partners differ from their base
    in dimensions 0 and 1 only; every coordinate stays in [0.5, 1), where the
    float spacing is 2^-24, so every difference is exact."""
    T = np.float32(oracle.sq_threshold(eps, np.float32))
    targets = [T, np.nextafter(T, np.float32(0)), np.nextafter(T, np.float32(np.inf))]
    u = np.float64(2.0 ** -24)
    rows, expect = [], []
    guard = np.full(d, 0.5, np.float32)              # the minimum corner: no real point gets cell coordinate 0
    rows.append(guard)
    for i in range(n_base):
        p = np.float32(0.62) + np.float32(0.25) * rng.random(d).astype(np.float32)
        p[:2] = np.float32(0.6) + np.float32(0.05) * np.float32(rng.random(2))
        p = p.astype(np.float32)
        tgt = targets[i % 3]
        # a: largest multiple of 2^-24 whose square rounds below the target; b tops it up exactly
        ka = int(np.floor(np.sqrt(np.float64(tgt)) / u)) - int(rng.integers(1, 30))
        acc0 = np.float32(np.float64(ka * u) ** 2)
        # fma(b, b, acc0) for b = j 2^-24: the sum is exact in FP64 (about 40 bits), then one rounding
        js = np.arange(0, 60000, dtype=np.float64)
        sums = ((js * u) ** 2 + np.float64(acc0)).astype(np.float32)
        hit = np.flatnonzero(sums == tgt)
        if len(hit) == 0:
            continue
        found = int(hit[0])
        c = p.copy()
        c[0] = np.float32(np.float64(p[0]) + ka * u)
        c[1] = np.float32(np.float64(p[1]) + found * u)
        assert oracle.sqdist(c, p, 1) == tgt and oracle.sqdist(p, c, 1) == tgt
        rows += [p, c]
        expect.append((len(rows) - 2, len(rows) - 1, tgt <= T))
    return np.array(rows, np.float32), expect


@pytest.mark.parametrize("d", [2, 18, 32])
def test_ties_at_threshold(cuda, d):
    rng = np.random.default_rng(62 + d)
    eps = np.float32(0.05)
    db, expect = _tie_dataset(d, eps, rng)
    assert len(expect) > 60
    kinds = ("exact",) if d < 16 else ("exact", "auto", "tc_f16", "tc_bf16")
    off, vals, _ = _check_all_kinds(db, 2 if d == 2 else 6, eps, cuda, kinds)
    for a, b, inside in expect:
        nb = set(vals[off[a]:off[a + 1]].tolist())
        assert (b in nb) == bool(inside)


def test_band_pairs_at_largest_norms(cuda):
    """Pairs spread over d^2 in [0.7 T, 1.3 T] around points at the far corner of
    the data (the largest |x - min|, where |q|^2 + |c|^2 - 2 q.c cancels most)."""
    import hegjoin_b200 as hj
    rng = np.random.default_rng(63)
    d, k, eps = 18, 6, np.float32(0.05)
    T = float(oracle.sq_threshold(eps, np.float32))
    bulk = workloads.exp40(63, 2000, d, np.float32)
    base = (np.float32(0.8) + np.float32(0.15) * rng.random((600, d))).astype(np.float32)
    dirs = rng.standard_normal((600, 3, d))
    dirs /= np.linalg.norm(dirs, axis=-1, keepdims=True)
    r = np.sqrt(T * rng.uniform(0.7, 1.3, (600, 3, 1)))
    partners = (base[:, None, :].astype(np.float64) + r * dirs).astype(np.float32).reshape(-1, d)
    db = np.concatenate([bulk, base, np.clip(partners, 0, np.float32(0.9999))]).astype(np.float32)
    ix, mn, nc = _index(db, k, eps, cuda)
    off, vals = oracle.join(db, k, eps, mn, nc)
    for refine in ("tc_f16", "tc_bf16"):
        res = hj.join(ix, refine=refine)
        goff, gvals = _csr(res)
        assert np.array_equal(goff, off) and np.array_equal(gvals, vals), refine
        assert res.stats.band_pairs > 0


def test_auto_falls_back_when_band_is_wide(cuda):
    """With eps tiny against the data's spread, FP16 quantisation error is a large
    fraction of eps: auto takes the exact path, and the explicit filter still
    returns the oracle's set (through a wide band)."""
    import hegjoin_b200 as hj
    db = workloads.exp40(64, 4000, 18, np.float32)
    corner = np.full((1, 18), 0.99, np.float32)      # the largest norm: quantisation error ~1e-3
    spread = np.concatenate([db, db[:200] + np.float32(1e-4), corner]).astype(np.float32)
    eps = np.float32(3e-4)
    _, _, used = _check_all_kinds(spread, 3, eps, cuda)
    assert used["auto"] == hj.HJ_REFINE_EXACT
    assert used["tc_f16"] == hj.HJ_REFINE_TC_F16
