"""The streamed join (hj_join_stream): nothing is kept on the device, every
grouped batch goes to a sink, and per-query digests accumulate on the device.

Its batches, concatenated, must be exactly the oracle's pair set (each query's
list whole within one batch), its digests must equal the retained join's, and
a sink that reports an error must stop the join cleanly.
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
    return hj.GridIndex(torch.from_numpy(db).to(dev), k, float(eps), [float(x) for x in mn],
                        [int(x) for x in nc]), mn, nc


@pytest.mark.parametrize("dtype,d,k,eps,refine", [(np.float64, 2, 2, 0.01, "exact"), (np.float32, 18, 6, 0.09, "auto"),
                                                  (np.float32, 6, 6, 0.04, "exact")])
def test_stream_batches_equal_oracle(cuda, dtype, d, k, eps, refine):
    import torch
    import hegjoin_b200 as hj
    db = workloads.exp40(80, 20000, d, dtype)
    ix, mn, nc = _index(db, k, eps, cuda)
    off, vals = oracle.join(db, k, eps, mn, nc)
    total = int(off[-1])
    got_k, got_v, seen = [], [], []

    def sink(batch, count, keys, vals_p, stream):
        seen.append((batch, count))
        if count:
            got_k.append(hj.device_view(keys, (count,), np.uint32).cpu().numpy().copy())
            got_v.append(hj.device_view(vals_p, (count,), np.uint32).cpu().numpy().copy())

    st, (c, s, x) = hj.join_stream(ix, sink, refine=refine, result_capacity=max(1, total // 6))
    assert st.total_pairs == total and st.n_batches > 1
    assert [b for b, _ in seen] == list(range(st.n_batches))
    assert sum(n for _, n in seen) == total
    keys = np.concatenate(got_k)
    v = np.concatenate(got_v)
    # every query's neighbours arrive in one batch; rebuild the CSR and compare
    order = np.lexsort((v, keys))
    keys, v = keys[order], v[order]
    goff = np.zeros(len(db) + 1, np.uint64)
    np.cumsum(np.bincount(keys, minlength=len(db)), out=goff[1:])
    assert np.array_equal(goff, off) and np.array_equal(v, vals)
    for batch_keys in got_k:
        assert (np.diff(batch_keys.astype(np.int64)) >= 0).all()     # grouped by query id
    # digests accumulated over the batches equal the retained join's
    res = hj.join(ix, refine=refine)
    for a, b in zip((c, s, x), res.digest()):
        assert torch.equal(a, b)
    oc, osum, oxor = oracle.digest(off, vals)
    assert np.array_equal(c.cpu().numpy().astype(np.uint32), oc)
    assert np.array_equal(s.cpu().numpy().view(np.uint64), osum)
    assert np.array_equal(x.cpu().numpy().view(np.uint64), oxor)


def test_stream_without_sink_and_sink_error(cuda):
    import torch
    import hegjoin_b200 as hj
    db = workloads.exp40(81, 10000, 2, np.float64)
    ix, mn, nc = _index(db, 2, 0.01, cuda)
    st, dig = hj.join_stream(ix, None, refine="exact")
    assert st.total_pairs == hj.join(ix, refine="exact").total_pairs
    torch.cuda.synchronize()
    base = hj.debug_pool_used()

    def failing(batch, count, keys, vals, stream):
        return hj.HJ_ERR_CUDA if batch == 1 else hj.HJ_OK

    with pytest.raises(hj.HJError) as e:
        hj.join_stream(ix, failing, refine="exact", result_capacity=st.total_pairs // 5)
    assert e.value.status == hj.HJ_ERR_CUDA and "sink" in str(e.value)
    torch.cuda.synchronize()
    assert hj.debug_pool_used() == base


@pytest.mark.parametrize("refine", ["exact", "auto"])
def test_stream_overlap_sink_on_its_own_stream(cuda, refine):
    """With stream_overlap, a sink that reads each batch on a stream of its own (after
    waiting for the batch on the join's stream) and hands back an event gets every batch
    intact, although the next batches run meanwhile."""
    import torch
    import hegjoin_b200 as hj
    d, k, eps, dtype = (2, 2, 0.01, np.float64) if refine == "exact" else (18, 6, 0.09, np.float32)
    db = workloads.exp40(82, 20000, d, dtype)
    ix, mn, nc = _index(db, k, eps, cuda)
    off, vals = oracle.join(db, k, eps, mn, nc)
    total = int(off[-1])
    side = torch.cuda.Stream()
    keep, events = [], []

    def sink(batch, count, keys, vals_p, stream):
        ready = torch.cuda.Event()
        ready.record(torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream())
        side.wait_event(ready)
        with torch.cuda.stream(side):
            # a slow reader: copies made on the side stream, after some unrelated work
            pad = torch.ones(1 << 22, device=cuda)
            for _ in range(20):
                pad = pad * 1.0001
            if count:
                keep.append((hj.device_view(keys, (count,), np.uint32).clone(),
                             hj.device_view(vals_p, (count,), np.uint32).clone()))
        done = torch.cuda.Event()
        done.record(side)
        events.append((ready, done, pad))
        return 0, done.cuda_event

    st, _ = hj.join_stream(ix, sink, refine=refine, result_capacity=max(1, total // 7), stream_overlap=True)
    torch.cuda.synchronize()
    assert st.total_pairs == total and st.n_batches > 2
    keys = np.concatenate([a.cpu().numpy() for a, _ in keep])
    v = np.concatenate([b.cpu().numpy() for _, b in keep])
    order = np.lexsort((v, keys))
    keys, v = keys[order], v[order]
    goff = np.zeros(len(db) + 1, np.uint64)
    np.cumsum(np.bincount(keys, minlength=len(db)), out=goff[1:])
    assert np.array_equal(goff, off) and np.array_equal(v, vals)
