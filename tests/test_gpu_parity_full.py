"""Parity at the configurations' stated sizes.

The 18-D (5,000,000 points), 90-D (500,000) and skewed 6-D (10,000,000) self
joins run on the GPU at full size.  The oracle then recomputes, for a seeded
sample of about 2,000 query points, their complete neighbour lists against the
whole dataset: the heaviest 300 and the lightest 700 of the workload order,
700 around its median, and 300 at random.  Counts and sorted lists must match
bit for bit under the default refine and the exact one.
"""
import hashlib
import json
import os
import time

import numpy as np
import pytest

import oracle
from hegjoin_b200 import workloads

pytestmark = pytest.mark.gpu


def _sample_queries(origin: np.ndarray, seed: int) -> np.ndarray:
    n = len(origin)
    rng = np.random.default_rng(seed)
    mid = n // 2
    picks = [origin[:300], origin[max(0, mid - 350):mid + 350], origin[max(0, n - 700):],
             rng.choice(n, 300, replace=False).astype(np.uint32)]
    return np.unique(np.concatenate(picks).astype(np.uint32))


def _gather_lists(off_d, vals_d, qids: np.ndarray):
    """Concatenated neighbour lists of qids (in that order) from a device CSR."""
    import torch
    q = torch.from_numpy(qids.astype(np.int64)).to(off_d.device)
    starts = off_d[q]
    lens = off_d[q + 1] - starts
    total = int(lens.sum().item())
    if total == 0:
        return lens.cpu().numpy(), np.zeros(0, np.uint32)
    base = torch.repeat_interleave(starts, lens)
    first = torch.repeat_interleave(torch.cumsum(lens, 0) - lens, lens)
    idx = base + torch.arange(total, device=off_d.device) - first
    return lens.cpu().numpy(), vals_d[idx].cpu().numpy().astype(np.uint32)


@pytest.mark.parametrize("name,refines", [("c2_18d", ("auto", "exact")), ("c3_90d", ("auto", "exact")),
                                          ("c4_skew6d", ("auto",))])
def test_full_size_sampled_lists_match_oracle(cuda, name, refines):
    import torch
    import hegjoin_b200 as hj
    wl = workloads.WORKLOADS[name]
    db = wl.generate()
    t0 = time.time()
    ix = hj.GridIndex(torch.from_numpy(db).to(cuda), wl.k, wl.eps)
    ix.sort_by_workload()
    _, origin = ix.workload_export()
    qids = _sample_queries(origin.cpu().numpy().astype(np.uint32), seed=wl.seed)
    mn, _, nc, _ = hj.grid_geometry(ix.db, wl.k, wl.eps)
    omn, _, onc, _ = oracle.geometry(db, wl.k, wl.eps)
    assert np.array_equal(np.array(mn, db.dtype), omn) and list(nc) == onc.tolist()
    counts, lists = oracle.join_lists(db, wl.k, wl.eps, qids, omn, onc)
    t_oracle = time.time() - t0
    totals = {}
    for refine in refines:
        res = hj.join(ix, refine=refine)
        off_d, vals_d = res.to_csr(sort_lists=True)
        gcounts, glists = _gather_lists(off_d, vals_d, qids)
        assert np.array_equal(gcounts.astype(np.uint32), counts), (name, refine)
        assert np.array_equal(glists, lists), (name, refine)
        totals[refine] = res.total_pairs
        print(f"{name} {refine}: {res.total_pairs} pairs, refine {res.stats.refine_used}, "
              f"{len(qids)} sampled queries with {int(counts.sum())} neighbours match the oracle")
        del off_d, vals_d
        res.close()
    assert len(set(totals.values())) == 1
    print(f"{name}: oracle sample {t_oracle:.1f} s")
    ix.close()


def test_c1_full_size_streamed_matches_oracle(cuda):
    """The 2-D FP64 configuration at 2,000,000 points (about 1.9e10 pairs, more than
    device memory holds) through the streamed join: every query's neighbour count
    equals the oracle's, and sampled queries' digests equal those of the oracle's
    neighbour lists."""
    import torch
    import hegjoin_b200 as hj
    wl = workloads.WORKLOADS["c1_2d"]
    db = wl.generate()
    ix = hj.GridIndex(torch.from_numpy(db).to(cuda), wl.k, wl.eps)
    ix.sort_by_workload()
    _, origin = ix.workload_export()
    qids = _sample_queries(origin.cpu().numpy().astype(np.uint32), seed=wl.seed)
    st, (c, s, x) = hj.join_stream(ix, None, digest=True, refine="exact")
    assert st.n_batches > 1
    # all 2M counts against the oracle's count pass (tests/golden/make_c1_counts.py)
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "c1_2d_counts.json")))
    assert (gold["n"], gold["eps"], gold["seed"]) == (wl.n, wl.eps, wl.seed)
    counts = c.cpu().numpy().astype("<u4")
    assert st.total_pairs == gold["total_pairs"]
    assert hashlib.sha256(counts.tobytes()).hexdigest() == gold["counts_sha256"]
    mn, _, nc, _ = oracle.geometry(db, wl.k, wl.eps)
    sc, lists = oracle.join_lists(db, wl.k, wl.eps, qids, mn, nc)
    soff = np.zeros(len(qids) + 1, np.uint64)
    np.cumsum(sc, out=soff[1:])
    _, osum, oxor = oracle.digest(soff, lists)
    q = torch.from_numpy(qids.astype(np.int64)).to(cuda)
    assert np.array_equal(s[q].cpu().numpy().view(np.uint64), osum)
    assert np.array_equal(x[q].cpu().numpy().view(np.uint64), oxor)
    print(f"c1_2d: {st.total_pairs} pairs in {st.n_batches} batches; all {len(db)} counts and "
          f"{len(qids)} sampled digests match the oracle")
    ix.close()
