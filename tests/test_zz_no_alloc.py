"""hj_grid_geometry_noalloc: the allocation-free geometry entry point.

It exists for callers that cannot allocate device memory at the point where
they need the grid geometry -- a process that reserves all of its device memory
up front and must not fail on an allocation later -- so its scratch is a static
device array shared by every call.  Called through the C ABI twice in
a row, on different data, it must return exactly what the allocating entry
point (hj_grid_geometry) returns: dataset-type minima and integer cell counts,
so the tolerance is zero.  k beyond the array's limit must be rejected.  This
file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fn(lib):
    P, U32, I, D = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_double
    f = lib.hj_grid_geometry_noalloc
    f.restype = I
    f.argtypes = [P, U32, U32, U32, I, D, P, P, P, P, P]
    return f


def _call(f, t, k, eps, dtype_code):
    n, d = t.shape
    mn = (ctypes.c_double * k)()
    mx = (ctypes.c_double * k)()
    nc = (ctypes.c_uint32 * k)()
    tot = ctypes.c_uint64()
    st = f(t.data_ptr(), n, d, k, dtype_code, float(eps), mn, mx, nc, ctypes.byref(tot), None)
    return st, list(mn), list(mx), list(nc), tot.value


@pytest.mark.parametrize("dtype,d,k,eps,n", [(np.float32, 18, 6, 0.0403, 200_000), (np.float64, 2, 2, 0.002, 300_000),
                                             (np.float32, 90, 16, 0.2, 5_000), (np.float32, 3, 3, 0.01, 7)])
def test_noalloc_geometry_matches_allocating_entry_point(cuda, dtype, d, k, eps, n):
    import torch
    import hegjoin_b200 as hj
    from hegjoin_b200 import workloads
    f = _fn(hj.lib)
    code = hj.HJ_F32 if dtype == np.float32 else hj.HJ_F64
    for seed in (1, 2):     # two calls in a row, on different data
        t = torch.from_numpy(workloads.exp40(seed, n, d, dtype)).to(cuda)
        ref = hj.grid_geometry(t, k, eps)
        st, mn, mx, nc, tot = _call(f, t, k, eps, code)
        assert st == hj.HJ_OK, hj.last_error()
        assert np.array_equal(np.array(mn), np.array(ref[0]))
        assert np.array_equal(np.array(mx), np.array(ref[1]))
        assert nc == list(ref[2]) and tot == ref[3]


def test_noalloc_rejects_k_beyond_limit(cuda):
    import torch
    import hegjoin_b200 as hj
    f = _fn(hj.lib)
    t = torch.rand((100, 20), device=cuda)
    st, *_ = _call(f, t, 17, 0.1, hj.HJ_F32)
    assert st == hj.HJ_ERR_INVALID
    assert "exceed" in hj.last_error()
