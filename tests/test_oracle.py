"""The CPU oracle (oracle/hj_oracle.cpp) against independent restatements.

The oracle is the checker for every GPU parity test, so it is itself checked
here: its squared distance against an exact rational evaluation of the fused
multiply-add chain, its grid index against a numpy restatement of GPU.cu:239-324,
and its join against a brute force over all pairs with the same cell rule.
"""
from fractions import Fraction

import numpy as np
import pytest

import oracle
from hegjoin_b200 import workloads


def _round_f32(fr: Fraction) -> np.float32:
    """Round a rational to the nearest float32, ties to even."""
    if fr == 0:
        return np.float32(0.0)
    sign = -1 if fr < 0 else 1
    fr = abs(fr)
    e = fr.numerator.bit_length() - fr.denominator.bit_length()
    if Fraction(2) ** e > fr:
        e -= 1
    e = max(e, -126)
    q = fr / (Fraction(2) ** (e - 23))          # 24-bit significand scale
    fl = q.numerator // q.denominator
    rem = q - fl
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and fl % 2 == 1):
        fl += 1
    return np.float32(sign * float(Fraction(fl) * Fraction(2) ** (e - 23)))


def _fma_chain_f32(c, q):
    acc = np.float32(0.0)
    for cl, ql in zip(c, q):
        diff = np.float32(np.float32(cl) - np.float32(ql))
        acc = _round_f32(Fraction(float(diff)) * Fraction(float(diff)) + Fraction(float(acc)))
    return acc


def test_sqdist_is_fma_chain():
    rng = np.random.default_rng(7)
    for d in (1, 2, 5, 18):
        for _ in range(200):
            a = rng.random(d, dtype=np.float32) * np.float32(rng.choice([1e-3, 1.0, 30.0]))
            b = rng.random(d, dtype=np.float32)
            got = np.float32(oracle.sqdist(a, b, 1))
            assert got == _fma_chain_f32(a, b), (d, a, b)


def test_sqdist_unfused_mode_differs_somewhere():
    rng = np.random.default_rng(3)
    diffs = 0
    for _ in range(2000):
        a = rng.random(18, dtype=np.float32)
        b = rng.random(18, dtype=np.float32)
        diffs += oracle.sqdist(a, b, 1) != oracle.sqdist(a, b, 0)
    assert diffs > 0


def test_threshold_matches_sqrt_rule():
    for eps in (0.002, 0.038387289, 0.2, 1e-7, 0.5):
        for dt in (np.float32, np.float64):
            t = oracle.sq_threshold(eps, dt)
            e = dt(eps)
            assert np.sqrt(t) <= e
            assert np.sqrt(np.nextafter(t, dt(np.inf))) > e


def _np_cells(db, k, eps, mn):
    t = db.dtype.type
    a = (db[:, :k] - mn.astype(db.dtype)).astype(db.dtype)
    c = (a / t(eps)).astype(db.dtype)
    return np.trunc(c).astype(np.uint64)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_geometry_and_index_restated(dtype):
    db = workloads.exp40(11, 3000, 4, dtype)
    k, eps = 3, 0.01
    mn, mx, nc, tot = oracle.geometry(db, k, eps)
    t = np.dtype(dtype).type
    assert np.array_equal(mn, (db[:, :k].min(0) - t(eps)).astype(dtype))
    assert np.array_equal(mx, (db[:, :k].max(0) + t(eps)).astype(dtype))
    assert np.array_equal(nc, np.ceil(((mx - mn) / t(eps)).astype(dtype)).astype(np.uint32))
    assert tot == int(np.prod(nc.astype(np.uint64)))
    lid, first, last, lookup = oracle.index(db, k, eps, mn, nc)
    coords = _np_cells(db, k, eps, mn)
    mult = np.cumprod(np.concatenate([[1], nc[:-1].astype(np.uint64)])).astype(np.uint64)
    plid = (coords * mult).sum(1).astype(np.uint64)
    order = np.argsort(plid, kind="stable")
    assert np.array_equal(lookup, order.astype(np.uint32))
    u, starts = np.unique(plid[order], return_index=True)
    assert np.array_equal(lid, u)
    assert np.array_equal(first, starts.astype(np.int32))
    assert np.array_equal(last, np.append(starts[1:] - 1, len(db) - 1).astype(np.int32))


def _brute(db, k, eps, mn, nc):
    """All pairs with the reference's cell rule and float64 distances."""
    coords = _np_cells(db, k, eps, mn).astype(np.int64)
    n = len(db)
    lo = coords - 1
    hi = np.minimum(nc.astype(np.int64) - 1, coords + 1)
    wrap = (coords == 0).any(1)
    inbox = np.ones((n, n), bool)
    for j in range(k):
        cj = coords[:, j]
        inbox &= (cj[None, :] >= lo[:, j][:, None]) & (cj[None, :] <= hi[:, j][:, None])
    inbox &= ~wrap[:, None]
    d2 = ((db[None, :, :].astype(np.float64) - db[:, None, :].astype(np.float64)) ** 2).sum(-1)
    return inbox, d2


@pytest.mark.parametrize("dtype,d,k,eps", [(np.float32, 2, 2, 0.01), (np.float32, 6, 3, 0.05),
                                           (np.float64, 2, 2, 0.004), (np.float32, 18, 6, 0.04)])
def test_join_against_brute_force(dtype, d, k, eps):
    db = workloads.exp40(5, 700, d, dtype)
    mn, _, nc, _ = oracle.geometry(db, k, eps)
    off, vals = oracle.join(db, k, eps, mn, nc)
    inbox, d2 = _brute(db, k, eps, mn, nc)
    thr = float(oracle.sq_threshold(eps, dtype))
    got = np.zeros_like(inbox)
    for q in range(len(db)):
        got[q, vals[off[q]:off[q + 1]]] = True
    sure_in = inbox & (d2 <= thr * (1 - 1e-5))
    sure_out = ~inbox | (d2 > thr * (1 + 1e-5))
    assert not (sure_out & got).any()
    assert (got | ~sure_in).all()
    assert got.sum() == off[-1] > len(db) // 2


def test_wrap_at_coordinate_zero_emits_nothing():
    # eps chosen so (min - (min - eps)) / eps rounds below 1 for the minimum point
    db = np.array([[0.7, 0.2], [0.7005, 0.2], [0.3, 0.9]], np.float32)
    found = False
    for e in np.linspace(0.001, 0.01, 400, dtype=np.float32):
        mn, _, nc, _ = oracle.geometry(db, 2, e)
        c = _np_cells(db, 2, e, mn)
        if (c == 0).any():
            found = True
            off, vals = oracle.join(db, 2, e, mn, nc)
            for q in range(3):
                if (c[q] == 0).any():
                    assert off[q + 1] == off[q]        # not even the self pair
            break
    assert found


def test_tie_exactly_at_threshold():
    eps = np.float32(0.25)
    db = np.array([[0.5, 0.5], [0.5, 0.75], [0.5, 0.7500001]], np.float32)
    off, vals = oracle.join(db, 2, eps)
    nb0 = set(vals[off[0]:off[1]].tolist())
    assert 1 in nb0 and 2 not in nb0 and 0 in nb0


def test_digest_order_independent():
    off = np.array([0, 3, 3, 5], np.uint64)
    v1 = np.array([5, 1, 9, 2, 4], np.uint32)
    v2 = np.array([9, 5, 1, 4, 2], np.uint32)
    a, b = oracle.digest(off, v1), oracle.digest(off, v2)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
