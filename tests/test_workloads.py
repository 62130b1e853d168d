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


def _mix64(z):
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def test_generator_definition():
    """The native generator follows its documented formula (checked through
    float32 outputs, where libm ulp differences rarely survive the cast)."""
    seed, n, d = 5, 400, 7
    got = workloads.exp40(seed, n, d, np.float32)
    salt = np.uint64(0xD1B54A32D192ED03)
    base = _mix64(np.array([np.uint64(seed) ^ salt], np.uint64))[0]
    with np.errstate(over="ignore"):
        z = _mix64(base + np.arange(n * d, dtype=np.uint64) * np.uint64(64))
    u = (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    exp = (-np.log1p(-u) / 40.0).astype(np.float32).reshape(n, d)
    assert (got == exp).mean() > 0.999
