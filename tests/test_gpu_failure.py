"""Failure detection and clean-up, in forms that cannot fault a GPU.

* A bounded wait of the tensor-core pipeline is made to run out (the tile probe
  issues no MMA and no commit after its loads have landed): the call reports
  HJ_ERR_TIMEOUT, the kernel releases its tensor memory, and the next join on
  the same context matches the oracle.
* Every device allocation of the index build, workload order and join is made
  to fail in turn (host-side fault injection): each attempt returns
  HJ_ERR_OOM and leaves the memory pool exactly as it found it.
* Two shards of one join (two ranks' work on one GPU) together give the
  unsharded pair set, each pair once.
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
    return hj.GridIndex(torch.from_numpy(db).to(dev), k, float(eps), [float(x) for x in mn], [int(x) for x in nc])


def _csr(res):
    off, vals = res.to_csr(sort_lists=True)
    return off.cpu().numpy().astype(np.uint64), vals.cpu().numpy().astype(np.uint32)


def test_tc_bounded_wait_expires_and_context_recovers(cuda):
    import hegjoin_b200 as hj
    db = workloads.exp40(70, 3000, 18, np.float32)
    ix = _index(db, 6, 0.07, cuda)
    for kind in ("tc_f16", "tc_bf16"):
        st = hj.lib.hj_probe_tc_wait_timeout(ix.handle, hj.REFINE_NAMES[kind], 2_000_000, None)
        assert st == hj.HJ_ERR_TIMEOUT, hj.last_error()
        assert "bounded wait" in hj.last_error()
    # tensor memory was released and the context is healthy: the filter runs again
    res = hj.join(ix, refine="tc_f16")
    off, vals = oracle.join(db, 6, 0.07)
    goff, gvals = _csr(res)
    assert np.array_equal(goff, off) and np.array_equal(gvals, vals)
    acc, _, _ = hj.probe_tc_tile(ix, "tc_f16", 0, 0)
    assert np.isfinite(acc).all()


def _pipeline(db, k, eps, refine, dev, **kw):
    import torch
    import hegjoin_b200 as hj
    ix = hj.GridIndex(torch.from_numpy(db).to(dev), k, float(eps))
    try:
        ix.sort_by_workload()
        res = hj.join(ix, refine=refine, **kw)
        n = res.total_pairs
        res.close()
        return n
    finally:
        ix.close()


@pytest.mark.parametrize("d,k,eps,refine,kw", [(18, 6, 0.07, "auto", {}), (2, 2, 0.01, "exact", {}),
                                               (2, 2, 0.01, "exact", {"result_capacity": 20000})])
def test_every_allocation_failure_is_clean(cuda, d, k, eps, refine, kw):
    import torch
    import hegjoin_b200 as hj
    db = workloads.exp40(71, 6000, d, np.float32)
    expect = _pipeline(db, k, eps, refine, cuda, **kw)       # also warms tuning and the pool
    torch.cuda.synchronize()
    base = hj.debug_pool_used()
    failures = 0
    for nth in range(1, 400):
        hj.debug_fail_alloc(nth)
        try:
            got = _pipeline(db, k, eps, refine, cuda, **kw)
            ok = True
        except hj.HJError as e:
            assert e.status == hj.HJ_ERR_OOM, str(e)
            assert "injected" in str(e)
            ok = False
        finally:
            hj.debug_fail_alloc(0)
        torch.cuda.synchronize()
        assert hj.debug_pool_used() == base, (nth, hj.debug_pool_used() - base)
        if ok:
            assert got == expect
            break
        failures += 1
    assert failures > 20                          # every allocation point was exercised
    assert _pipeline(db, k, eps, refine, cuda, **kw) == expect


@pytest.mark.parametrize("d,k,eps,refine", [(18, 6, 0.06, "auto"), (2, 2, 0.01, "exact"), (6, 6, 0.05, "exact")])
def test_two_shards_give_the_whole_join_once(cuda, d, k, eps, refine):
    import hegjoin_b200 as hj
    db = workloads.exp40(72, 20000, d, np.float32)
    ix = _index(db, k, eps, cuda)
    full = hj.join(ix, refine=refine)
    foff, fvals = _csr(full)
    parts = []
    for r in range(2):
        res = hj.join(ix, refine=refine, shard_count=2, shard_index=r)
        parts.append(_csr(res))
        assert 0 < res.total_pairs < full.total_pairs
    assert sum(int(p[0][-1]) for p in parts) == full.total_pairs
    # a query's work item belongs to one shard: its whole list is in exactly one part
    for q in range(len(db)):
        lists = [p[1][p[0][q]:p[0][q + 1]] for p in parts]
        nonempty = [l for l in lists if len(l)]
        assert len(nonempty) <= 1
        want = fvals[foff[q]:foff[q + 1]]
        got = nonempty[0] if nonempty else np.zeros(0, np.uint32)
        assert np.array_equal(got, want)
