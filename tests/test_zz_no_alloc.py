"""pb_morton_sort_noalloc against the regular build entry point.

The no-allocation variant serves callers that cannot call cudaMalloc (applications that
own all device memory through their own pool, or pipelines that cannot take an
allocation's synchronisation).  Its scratch is a fixed static device array shared by all
calls, so this test makes two calls in a row with different data and sizes and checks
that each one reproduces, bit for bit, the Morton codes and sorting order that
pb_linear_bvh + pb_export_encoding produce for the same particles -- at the largest size
it accepts too -- that a size above the limit is refused, and that a non-finite
coordinate is reported without spoiling the next call.  It runs last (file name) so a failure here leaves every other GPU
test already run; it passes both alone and after the other tests.
"""
import ctypes

import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_N = 262144


def _regular(backend, x, y, z):
    n = len(x)
    one = np.ones(n)
    inp = pb.InterpolationInput(x.copy(), y.copy(), z.copy(), one.copy(), one.copy(), one.copy(), ())
    lb = pb.LinearBVH_build(inp, backend, permute_input=False)
    return lb.encoding()


def _noalloc(lib, x, y, z):
    import torch
    n = len(x)
    dx, dy, dz = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (x, y, z))
    codes = torch.empty(n, dtype=torch.int64, device="cuda")
    order = torch.empty(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.pb_morton_sort_noalloc(dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), n, codes.data_ptr(),
                                    order.data_ptr(), None)
    return rc, codes.cpu().numpy().view(np.uint64), order.cpu().numpy()


def test_noalloc_matches_regular_build_twice():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    lib = _lib.load()
    backend = pb.CUDAComputeBackend(0)
    g = np.random.default_rng(42)
    cases = [g.normal(0, 10, (3, 200003)), g.integers(0, 4, (3, 5000)) / 3.0]   # second: many duplicate codes
    for pts in cases:
        x, y, z = (np.ascontiguousarray(a, np.float64) for a in pts)
        rc, codes, order = _noalloc(lib, x, y, z)
        assert rc == _lib.PB_OK
        exp_codes, exp_order = _regular(backend, x, y, z)
        assert np.array_equal(codes, exp_codes)
        assert np.array_equal(order, exp_order)
    backend.close()


def test_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    n = MAX_N + 1
    t = torch.zeros(n, dtype=torch.float64, device="cuda")
    out = torch.empty(n, dtype=torch.int64, device="cuda")
    rc = lib.pb_morton_sort_noalloc(t.data_ptr(), t.data_ptr(), t.data_ptr(), n, out.data_ptr(), out.data_ptr(), None)
    assert rc == _lib.PB_ERR_CAPACITY


def test_noalloc_at_the_size_limit_then_nonfinite_then_again():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    backend = pb.CUDAComputeBackend(0)
    g = np.random.default_rng(7)
    x, y, z = (np.ascontiguousarray(a) for a in g.uniform(-50, 50, (3, MAX_N)))
    rc, codes, order = _noalloc(lib, x, y, z)
    assert rc == _lib.PB_OK
    exp_codes, exp_order = _regular(backend, x, y, z)
    assert np.array_equal(codes, exp_codes) and np.array_equal(order, exp_order)
    bad = x[:1000].copy()
    bad[123] = np.nan
    rc, _, _ = _noalloc(lib, bad, y[:1000], z[:1000])
    assert rc == _lib.PB_ERR_INVALID
    # the status word is cleared by the next call, which succeeds
    rc, codes, order = _noalloc(lib, x[:1000], y[:1000], z[:1000])
    assert rc == _lib.PB_OK
    exp_codes, exp_order = _regular(backend, x[:1000], y[:1000], z[:1000])
    assert np.array_equal(codes, exp_codes) and np.array_equal(order, exp_order)
    # host memory is refused (the caller must pass device pointers)
    out = np.empty(10, np.int64)
    h = np.zeros(10)
    assert lib.pb_morton_sort_noalloc(h.ctypes.data, h.ctypes.data, h.ctypes.data, 10, out.ctypes.data,
                                      out.ctypes.data, None) == _lib.PB_ERR_INVALID
    backend.close()
