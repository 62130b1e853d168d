"""Seeded synthetic workloads for the epsilon self-join.

The reference ships a generator (datasets/dataset_gen_fixed_len_expo_dist.cpp:24-91)
that draws each coordinate i.i.d. from Exp(rate=40) with ``std::mt19937`` and
redraws values above 1.  The workloads here keep that distribution but use a
counter-based generator, so any slice of a dataset can be produced in parallel
and reproduced bit for bit; its definition is hegjoin_b200/csrc/hj_datagen.cpp
(host C++, its own library libhj_datagen.so):

    u(seed, i, a) = (mix64(mix64(seed ^ SALT ^ K*stream) + 64*i + a) >> 11) * 2**-53   in [0, 1)
    x = -log1p(-u) / 40        (float64), cast to the dataset dtype,
    attempt a = 0, 1, ... until the cast value is < 1.

``i`` is the flat coordinate index (point * d + dim).  The Gaussian-cluster part
of the skewed workload uses Box-Muller on two further streams.

Each workload names its shape (n, d, k, dtype), seed and epsilon; epsilon for
the calibrated workloads is the value found by ``calibrate_eps`` on a seeded 1%
query sample (stored to 17 significant digits in EPS_TABLE).
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

# The generator is its own host library (libhj_datagen.so, declared in
# include/hegjoin_datagen.h): this module needs neither a GPU nor the join's
# CUDA library, so a process timing a CPU join can make the same inputs.
_DATAGEN_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libhj_datagen.so")
_dg = None


def _datagen():
    global _dg
    if _dg is None:
        if not os.path.exists(_DATAGEN_PATH):
            raise ImportError(f"{_DATAGEN_PATH} is missing: build it with `make -C hegjoin_b200/csrc`")
        lib = ctypes.CDLL(_DATAGEN_PATH)
        U32, U64, I, D, P = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double, ctypes.c_void_p
        lib.hj_generate_exp40.argtypes = [U64, U64, U64, U32, I, P]
        lib.hj_generate_exp40.restype = I
        lib.hj_generate_skewed.argtypes = [U64, U64, U32, U32, D, D, I, P]
        lib.hj_generate_skewed.restype = I
        _dg = lib
    return _dg


def _code(dtype) -> int:
    return 0 if np.dtype(dtype) == np.float32 else 1


def exp40(seed: int, n: int, d: int, dtype=np.float32, stream: int = 0) -> np.ndarray:
    """n x d coordinates, i.i.d. Exp(rate=40) redrawn into [0, 1) after the dtype cast."""
    out = np.empty((n, d), dtype=dtype)
    st = _datagen().hj_generate_exp40(seed, stream, n, d, _code(dtype), out.ctypes.data)
    if st != 0:
        raise ValueError(f"hj_generate_exp40 failed ({st})")
    return out


def skewed(seed: int, n: int, d: int, n_clusters: int = 64, sigma: float = 0.002,
           frac_clustered: float = 0.2, dtype=np.float32) -> np.ndarray:
    """80% Exp(40) points and 20% from Gaussian clusters, clipped to [0, 1)."""
    out = np.empty((n, d), dtype=dtype)
    st = _datagen().hj_generate_skewed(seed, n, d, n_clusters, sigma, frac_clustered, _code(dtype), out.ctypes.data)
    if st != 0:
        raise ValueError(f"hj_generate_skewed failed ({st})")
    return out


@dataclasses.dataclass(frozen=True)
class Workload:
    name: str
    n: int
    d: int
    k: int
    dtype: str          # "f32" or "f64"
    seed: int
    eps: float          # epsilon in the dataset dtype (exactly representable)
    target_neighbours: float | None = None
    kind: str = "exp40"

    @property
    def np_dtype(self):
        return np.float32 if self.dtype == "f32" else np.float64

    def generate(self, n: int | None = None) -> np.ndarray:
        n = self.n if n is None else n
        if self.kind == "skewed":
            return skewed(self.seed, n, self.d, dtype=self.np_dtype)
        return exp40(self.seed, n, self.d, self.np_dtype)


# Epsilon values found by calibrate_eps (1% seeded query sample against the full
# dataset, bisection to the target mean neighbour count), as dataset-dtype values.
EPS_TABLE = {
    "c2_18d": 0.04033349081873894,     # mean 50.0003 neighbours on the sample
    "c3_90d": 0.20804697275161743,     # mean 30.0008
    "c4_skew6d": 0.003275492461398244,  # mean 200.18
}

WORKLOADS = {
    "c1_2d": Workload("c1_2d", 2_000_000, 2, 2, "f64", 0, 0.002),
    "c2_18d": Workload("c2_18d", 5_000_000, 18, 6, "f32", 1, EPS_TABLE["c2_18d"], 50.0),
    "c3_90d": Workload("c3_90d", 500_000, 90, 6, "f32", 2, EPS_TABLE["c3_90d"], 30.0),
    "c4_skew6d": Workload("c4_skew6d", 10_000_000, 6, 6, "f32", 3, EPS_TABLE["c4_skew6d"], 200.0, "skewed"),
}


def _sample_queries(n: int, sample_frac: float, seed: int) -> np.ndarray:
    m = max(1, int(n * sample_frac))
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=m, replace=False))


def _d2_histogram(x: np.ndarray, qi: np.ndarray, edges, device: str) -> np.ndarray:
    """Counts of (sampled query, point) squared distances per bin of `edges`."""
    import torch
    X = torch.from_numpy(x).to(device=device, dtype=torch.float32)
    Q = X[torch.from_numpy(qi).to(device)]
    E = torch.as_tensor(edges, dtype=torch.float32, device=device)
    hist = torch.zeros(len(edges) + 1, dtype=torch.int64, device=device)
    xn = (X * X).sum(1)
    chunk = max(1, int(2e8 // x.shape[0]))
    for s in range(0, len(qi), chunk):
        q = Q[s:s + chunk]
        d2 = (q * q).sum(1)[:, None] + xn[None, :] - 2.0 * (q @ X.T)
        d2.clamp_(min=0)
        hist += torch.bincount(torch.bucketize(d2.reshape(-1), E), minlength=len(edges) + 1)
    return hist.cpu().numpy()


def calibrate_eps(x: np.ndarray, target: float, sample_frac: float = 0.01, seed: int = 12345,
                  device: str = "cuda") -> float:
    """Epsilon whose mean neighbour count (self included) over a seeded 1% query
    sample, counted against the full dataset, first reaches `target`.

    Two histogram passes on the GPU: log-spaced bins over d2, then linear bins
    inside the bin where the mean crosses the target.  Returned as the dataset's
    float32 value.
    """
    qi = _sample_queries(x.shape[0], sample_frac, seed)
    m = len(qi)
    edges = np.geomspace(1e-10, 4.0 * x.shape[1], 4000)
    h = _d2_histogram(x, qi, edges, device)
    cum = np.cumsum(h)[:-1] / m            # mean count with d2 <= edges[i]
    i = int(np.searchsorted(cum, target))
    lo = edges[i - 1] if i > 0 else 0.0
    hi = edges[min(i, len(edges) - 1)]
    fine = np.linspace(lo, hi, 2001)
    h2 = _d2_histogram(x, qi, fine, device)
    base = cum[i - 1] if i > 0 else 0.0
    cum2 = base + np.cumsum(h2)[:-1] / m - (np.sum(h2[:1]) / m if i > 0 else 0.0)
    j = min(int(np.searchsorted(cum2, target)), len(fine) - 1)
    return float(np.float32(np.sqrt(fine[j])))


def mean_neighbours_sample(x: np.ndarray, eps: float, sample_frac: float = 0.01, seed: int = 12345,
                           device: str = "cuda") -> float:
    qi = _sample_queries(x.shape[0], sample_frac, seed)
    h = _d2_histogram(x, qi, np.array([eps * eps]), device)
    return float(h[0]) / len(qi)


if __name__ == "__main__":
    import json
    import sys
    out = {}
    for name in sys.argv[1:]:
        w = WORKLOADS[name]
        x = w.generate()
        e = calibrate_eps(x, w.target_neighbours)
        out[name] = {"eps": e, "eps_repr": repr(e), "mean_neighbours": mean_neighbours_sample(x, e),
                     "target": w.target_neighbours}
        print(json.dumps({name: out[name]}), flush=True)
