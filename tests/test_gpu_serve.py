"""Serving loop: every request's result is the same alone and in the concurrent mix."""
import numpy as np
import pytest

from hegjoin_b200 import workloads

pytestmark = pytest.mark.gpu


def _requests():
    rng = np.random.default_rng(7)
    out = []
    for i in range(24):
        d = int(rng.choice([2, 6, 18, 32, 90]))
        n = int(np.exp(rng.uniform(np.log(1000), np.log(40000))))
        k = min(d, 6)
        eps = {2: 0.004, 6: 0.03, 18: 0.06, 32: 0.1, 90: 0.22}[d]
        out.append((workloads.exp40(1000 + i, n, d, np.float32), k, eps))
    return out


def _digest(res):
    c, s, x = res.digest()
    return c.cpu().numpy(), s.cpu().numpy(), x.cpu().numpy()


def test_alone_equals_in_the_mix(cuda):
    import hegjoin_b200 as hj
    reqs = _requests()
    alone = []
    for db, k, eps in reqs:
        srv = hj.Server(workers=1)
        t = srv.submit(db, k, eps)
        res, info = srv.wait(t)
        alone.append((_digest(res), res.total_pairs))
        srv.close()
    srv = hj.Server(workers=6, hbm_budget=8 << 30)
    tickets = [srv.submit(db, k, eps) for db, k, eps in reqs]
    overlap = 0
    infos = []
    for i, t in enumerate(tickets):
        res, info = srv.wait(t)
        infos.append(info)
        d, tot = alone[i]
        assert res.total_pairs == tot and tot >= len(reqs[i][0])
        for a, b in zip(_digest(res), d):
            assert np.array_equal(a, b)
    # requests really ran concurrently: some admitted before an earlier one finished
    for i in range(1, len(infos)):
        if infos[i].t_admit < max(x.t_done for x in infos[:i]):
            overlap += 1
    assert overlap > 0
    srv.close()


def test_budget_admits_in_order(cuda):
    import hegjoin_b200 as hj
    # a budget smaller than one request still runs requests, one at a time
    srv = hj.Server(workers=4, hbm_budget=1)
    reqs = _requests()[:6]
    tickets = [srv.submit(db, k, eps) for db, k, eps in reqs]
    infos = [srv.wait(t, keep_result=False)[1] for t in tickets]
    for a, b in zip(infos, infos[1:]):
        assert b.t_admit >= a.t_done - 1e-6
    srv.close()


def _oracle_digest(db, k, eps):
    import oracle
    mn, _, nc, _ = oracle.geometry(db, k, eps)
    off, vals = oracle.join(db, k, eps, mn, nc)
    return oracle.digest(off, vals)


def test_served_results_match_the_oracle(cuda):
    import hegjoin_b200 as hj
    reqs = _requests()[:12]
    srv = hj.Server(workers=6, hbm_budget=8 << 30)
    tickets = [srv.submit(db, k, eps) for db, k, eps in reqs]
    for (db, k, eps), t in zip(reqs, tickets):
        res, _ = srv.wait(t)
        got = _digest(res)
        want = _oracle_digest(db, k, eps)
        assert np.array_equal(got[0].astype(np.uint32), want[0])
        assert np.array_equal(got[1].view(np.uint64), want[1])
        assert np.array_equal(got[2].view(np.uint64), want[2])
    srv.close()


def _dense_request():
    # ~440 neighbours per point (13.3M pairs): several times the serving loop's first
    # allowance of 64 per point
    db = workloads.exp40(77, 30000, 6, np.float32)
    return db, 6, 0.025


def test_join_cap_refuses_then_fits(cuda):
    """hj_join under device_bytes_cap: refused with the bytes it wants, then run within
    them (and within a third of them, in more batches) with the same pairs; the pool's
    high-water mark over the capped join stays within the cap."""
    import torch
    import hegjoin_b200 as hj
    db, k, eps = _dense_request()
    ix = hj.GridIndex(torch.from_numpy(db).cuda(), k, eps)
    ix.sort_by_workload()
    free = hj.join(ix, refine="exact")
    ref = _digest(free)
    want_pairs = free.total_pairs
    del free
    with pytest.raises(hj.HJError) as e:
        hj.join(ix, refine="exact", device_bytes_cap=1 << 20)
    assert e.value.status == hj.HJ_ERR_OOM
    wanted = e.value.stats.bytes_wanted
    assert wanted > 4 * want_pairs
    for cap, more_batches in ((wanted, False), (wanted // 3, True)):
        torch.cuda.synchronize()
        base = hj.debug_pool_used()
        hj.debug_pool_peak(reset=True)
        res = hj.join(ix, refine="exact", device_bytes_cap=cap)
        torch.cuda.synchronize()
        peak = hj.debug_pool_peak()
        assert res.total_pairs == want_pairs
        assert res.stats.n_batches >= (2 if more_batches else 1)
        for a, b in zip(_digest(res), ref):
            assert np.array_equal(a, b)
        # the cap covers result buffers and kept results; the join's other temporaries
        # (work items, estimator samples, control block) are a few MB here
        assert peak - base <= cap + (8 << 20), (peak - base, cap)
        del res


def test_server_regrants_a_heavy_request(cuda):
    import hegjoin_b200 as hj
    db, k, eps = _dense_request()
    light = _requests()[:4]
    srv = hj.Server(workers=3, hbm_budget=6 << 30)
    t_heavy = srv.submit(db, k, eps)
    t_light = [srv.submit(x, kk, e) for x, kk, e in light]
    res, info = srv.wait(t_heavy)
    assert info.regrants >= 1 and info.reserved_bytes >= info.stats.bytes_wanted
    want = _oracle_digest(db, k, eps)
    got = _digest(res)
    assert np.array_equal(got[0].astype(np.uint32), want[0])
    assert np.array_equal(got[1].view(np.uint64), want[1])
    for t in t_light:
        srv.wait(t, keep_result=False)
    cur, peak = srv.usage()
    assert peak <= 6 << 30
    srv.close()
