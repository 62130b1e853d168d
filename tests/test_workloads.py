import numpy as np

from hegjoin_b200 import workloads


def test_exp40_deterministic_and_in_range():
    a = workloads.exp40(1, 1000, 18, np.float32)
    b = workloads.exp40(1, 1000, 18, np.float32)
    assert np.array_equal(a, b)
    assert a.dtype == np.float32 and a.shape == (1000, 18)
    assert (a >= 0).all() and (a < 1).all()
    assert abs(float(a.mean()) - 1 / 40) < 2e-3
    c = workloads.exp40(2, 1000, 18, np.float32)
    assert not np.array_equal(a, c)


def test_prefix_stable():
    # a smaller n is a prefix of the bigger dataset (flat coordinate counter)
    a = workloads.exp40(3, 500, 6, np.float64)
    b = workloads.exp40(3, 200, 6, np.float64)
    assert np.array_equal(a[:200], b)


def test_skewed_mix():
    x = workloads.skewed(3, 5000, 6)
    assert x.shape == (5000, 6) and (x >= 0).all() and (x < 1).all()
    tail = x[4000:]
    # clustered points sit in tight groups: many near-duplicates at the 0.01 scale
    q = np.floor(tail / 0.01)
    assert len(np.unique(q, axis=0)) < 0.5 * len(tail)
