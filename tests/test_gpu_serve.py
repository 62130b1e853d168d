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
