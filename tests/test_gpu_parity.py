"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Integer and index outputs are compared bit for bit; pair sets are compared as
per-query sorted neighbour lists (small sizes) or per-query order-independent
digests (medium sizes).
"""
import numpy as np
import pytest

import oracle
from hegjoin_b200 import workloads

pytestmark = pytest.mark.gpu

CASES = [
    # dtype, n, d, k, eps
    (np.float32, 4000, 2, 2, 0.01),
    (np.float64, 4000, 2, 2, 0.004),
    (np.float32, 3000, 6, 6, 0.06),
    (np.float32, 2500, 18, 6, 0.06),
    (np.float32, 1500, 90, 6, 0.25),
    (np.float32, 2000, 5, 3, 0.05),
    (np.float64, 1500, 6, 4, 0.06),
    (np.float32, 1200, 32, 6, 0.12),
]


def _to_dev(db, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(db)).to(dev)


def _gpu_index(db, k, eps, dev):
    import hegjoin_b200 as hj
    mn, _, nc, _ = oracle.geometry(db, k, eps)
    return hj.GridIndex(_to_dev(db, dev), k, float(eps), [float(x) for x in mn], [int(x) for x in nc]), mn, nc


@pytest.mark.parametrize("dtype,n,d,k,eps", CASES)
def test_geometry(cuda, dtype, n, d, k, eps):
    import hegjoin_b200 as hj
    db = workloads.exp40(21, n, d, dtype)
    mn, mx, nc, tot = oracle.geometry(db, k, eps)
    gmn, gmx, gnc, gtot = hj.grid_geometry(_to_dev(db, cuda), k, float(eps))
    assert np.array_equal(np.array(gmn, dtype=dtype), mn)
    assert np.array_equal(np.array(gmx, dtype=dtype), mx)
    assert list(gnc) == nc.tolist() and gtot == tot


@pytest.mark.parametrize("dtype,n,d,k,eps", CASES)
def test_index_bit_exact(cuda, dtype, n, d, k, eps):
    db = workloads.exp40(22, n, d, dtype)
    ix, mn, nc = _gpu_index(db, k, eps, cuda)
    lid, first, last, lookup = oracle.index(db, k, eps, mn, nc)
    glid, gfirst, glast, glookup, gidx = ix.export()
    assert ix.info().n_nonempty_cells == len(lid)
    assert np.array_equal(glid.cpu().numpy().astype(np.uint64), lid)
    assert np.array_equal(gfirst.cpu().numpy(), first)
    assert np.array_equal(glast.cpu().numpy(), last)
    assert np.array_equal(glookup.cpu().numpy().astype(np.uint32), lookup)
    assert np.array_equal(gidx.cpu().numpy(), np.arange(len(lid)))


@pytest.mark.parametrize("dtype,n,d,k,eps", CASES)
def test_workload_order(cuda, dtype, n, d, k, eps):
    db = workloads.exp40(23, n, d, dtype)
    ix, mn, nc = _gpu_index(db, k, eps, cuda)
    nb, total = oracle.cell_workload(db, k, eps, mn, nc)
    assert ix.sort_by_workload() == total
    sched, origin = ix.workload_export()
    sched = sched.cpu().numpy()
    # every cell once, with the oracle's candidate count, heaviest first, stable among equals
    assert np.array_equal(np.sort(sched[:, 1]), np.arange(len(nb)))
    assert np.array_equal(sched[:, 0], nb[sched[:, 1]].astype(np.int32))
    assert (np.diff(sched[:, 0]) <= 0).all()
    ties = np.diff(sched[:, 0]) == 0
    assert (np.diff(sched[:, 1])[ties] > 0).all()
    # originPointIndex: cells in that order, members in indexLookupArr order (SortByWorkload.cu:155-181)
    lid, first, last, lookup = oracle.index(db, k, eps, mn, nc)
    exp = np.concatenate([lookup[first[c]:last[c] + 1] for c in sched[:, 1]])
    assert np.array_equal(origin.cpu().numpy().astype(np.uint32), exp)


def _csr(res):
    off, vals = res.to_csr(sort_lists=True)
    return off.cpu().numpy().astype(np.uint64), vals.cpu().numpy().astype(np.uint32)


@pytest.mark.parametrize("dtype,n,d,k,eps", CASES)
def test_join_exact_matches_oracle(cuda, dtype, n, d, k, eps):
    import hegjoin_b200 as hj
    db = workloads.exp40(24, n, d, dtype)
    ix, mn, nc = _gpu_index(db, k, eps, cuda)
    res = hj.join(ix, refine="exact")
    off, vals = oracle.join(db, k, eps, mn, nc)
    goff, gvals = _csr(res)
    assert res.total_pairs == int(off[-1])
    assert np.array_equal(goff, off)
    assert np.array_equal(gvals, vals)


def test_join_digest_medium(cuda):
    import hegjoin_b200 as hj
    db = workloads.exp40(25, 60000, 6, np.float32)
    k, eps = 6, 0.03
    ix, mn, nc = _gpu_index(db, k, eps, cuda)
    res = hj.join(ix, refine="exact")
    off, vals = oracle.join(db, k, eps, mn, nc)
    cnt, s, x = oracle.digest(off, vals)
    gc, gs, gx = (t.cpu().numpy() for t in res.digest())
    assert np.array_equal(gc.astype(np.uint32), cnt)
    assert np.array_equal(gs.view(np.uint64), s)
    assert np.array_equal(gx.view(np.uint64), x)


def test_overflow_split_and_retry(cuda):
    import hegjoin_b200 as hj
    db = workloads.exp40(26, 20000, 2, np.float32)
    k, eps = 2, 0.01
    ix, mn, nc = _gpu_index(db, k, eps, cuda)
    ref = hj.join(ix, refine="exact")
    small = hj.join(ix, refine="exact", result_capacity=max(1, ref.total_pairs // 7))
    assert small.stats.n_batches > 1
    assert small.total_pairs == ref.total_pairs
    assert all(np.array_equal(a, b) for a, b in zip(_csr(small), _csr(ref)))


def test_underestimate_forces_retry(cuda):
    # a sample rate of 1/64 on clustered data under-predicts some batches; the
    # overflowing batch is split and re-run instead of writing out of bounds
    import hegjoin_b200 as hj
    db = workloads.skewed(27, 30000, 6)
    k, eps = 6, 0.02
    ix, mn, nc = _gpu_index(db, k, eps, cuda)
    ref = hj.join(ix, refine="exact")
    r = hj.join(ix, refine="exact", sample_rate=1 / 64, result_capacity=ref.total_pairs // 5)
    assert r.total_pairs == ref.total_pairs
    assert all(np.array_equal(a, b) for a, b in zip(_csr(r), _csr(ref)))


@pytest.mark.parametrize("n", [1, 2, 3, 33])
def test_tiny_inputs(cuda, n):
    import hegjoin_b200 as hj
    db = workloads.exp40(28, n, 3, np.float32)
    ix, mn, nc = _gpu_index(db, 2, 0.05, cuda)
    res = hj.join(ix, refine="exact")
    off, vals = oracle.join(db, 2, 0.05, mn, nc)
    goff, gvals = _csr(res)
    assert np.array_equal(goff, off) and np.array_equal(gvals, vals)


def test_duplicates_and_single_cell(cuda):
    import hegjoin_b200 as hj
    base = workloads.exp40(29, 50, 4, np.float32)
    db = np.repeat(base, 20, axis=0)           # every point 20 times
    for eps in (1e-4, 0.9):                    # many tiny cells / one huge cell
        ix, mn, nc = _gpu_index(db, 4, eps, cuda)
        res = hj.join(ix, refine="exact")
        off, vals = oracle.join(db, 4, eps, mn, nc)
        goff, gvals = _csr(res)
        assert np.array_equal(goff, off) and np.array_equal(gvals, vals)


def test_wrap_at_coordinate_zero(cuda):
    import hegjoin_b200 as hj
    db = np.array([[0.7, 0.2], [0.7005, 0.2], [0.3, 0.9], [0.70001, 0.2001]], np.float32)
    hit = 0
    for e in np.linspace(0.001, 0.01, 400, dtype=np.float32):
        mn, _, nc, _ = oracle.geometry(db, 2, e)
        coords = np.trunc(((db[:, :2] - mn) / e).astype(np.float32))
        if not (coords == 0).any():
            continue
        hit += 1
        ix, _, _ = _gpu_index(db, 2, e, cuda)
        res = hj.join(ix, refine="exact")
        off, vals = oracle.join(db, 2, e, mn, nc)
        goff, gvals = _csr(res)
        assert np.array_equal(goff, off) and np.array_equal(gvals, vals)
        if hit >= 5:
            break
    assert hit


def test_fma_contraction_probe(cuda):
    """nvcc's default build of kernel.cu:350-353 is the fused chain the oracle uses."""
    import hegjoin_b200 as hj
    rng = np.random.default_rng(5)
    for dtype in (np.float32, np.float64):
        a = rng.random((20000, 18)).astype(dtype)
        b = rng.random((20000, 18)).astype(dtype)
        got = hj.probe_sqdist(_to_dev(a, cuda), _to_dev(b, cuda)).cpu().numpy()
        fused = np.array([oracle.sqdist(b[i], a[i], 1) for i in range(len(a))], dtype)
        unfused = np.array([oracle.sqdist(b[i], a[i], 0) for i in range(len(a))], dtype)
        assert (fused != unfused).any()
        # probe computes (a - b)^2 which equals (b - a)^2 bit for bit
        assert np.array_equal(got, fused)


def test_host_entry_point(cuda):
    import hegjoin_b200 as hj
    db = workloads.exp40(30, 5000, 18, np.float32)
    res = hj.self_join_host(db, 6, 0.07, refine="exact")
    off, vals = oracle.join(db, 6, 0.07)
    goff, gvals = _csr(res)
    assert np.array_equal(goff, off) and np.array_equal(gvals, vals)
