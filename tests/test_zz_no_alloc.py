"""psb_reduce_noalloc: the allocation-free reduction entry point.

It exists for callers that are not allowed to call cudaMalloc -- a host
framework that owns all device memory through its own allocator and budget,
or a latency-critical loop where an allocation would synchronise the device.
It must give the same answer as the allocating entry point (psb_reduce), call
after call, while keeping its scratch in a fixed static device array.

This file is collected last on purpose, so a run that stops at the first
failure has already run every other test; it also passes alone in a fresh
process (it sets up its own grid).
"""
import ctypes

import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle

lib = ps.lib
lib.psb_reduce_noalloc.restype = ctypes.c_int
lib.psb_reduce_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_int64),
                                   ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p,
                                   ctypes.POINTER(ctypes.c_double)]


def _device_view(g):
    """Device pointer of element (0,0,0), extents and strides of a grid."""
    origin = ps.PSGridStruct.from_address(g.ptr.value).p0
    lay = g.layout()
    ext = (ctypes.c_int64 * 3)(*g.dims)
    strides = (ctypes.c_int64 * 2)(lay["stride_y"], lay["stride_z"])
    return origin, ext, strides


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_noalloc_matches_allocating_entry_point(dtype):
    a = (np.random.default_rng(41).random((37, 45, 131)) - 0.25).astype(dtype)
    t = ps.PS_FLOAT if dtype == np.float32 else ps.PS_DOUBLE
    g = ps.grid_new(t, (131, 45, 37))
    try:
        ps.PSGridCopyin(g, a)
        origin, ext, strides = _device_view(g)
        _, abssum = oracle.sum_f64(a)
        for op in (ps.PS_SUM, ps.PS_MAX, ps.PS_MIN, ps.PS_SUM):
            want = ps.reduce64(op, g)
            for call in range(2):  # two calls in a row share the static scratch
                got = ctypes.c_double()
                rc = lib.psb_reduce_noalloc(origin, t, op, ext, strides, None,
                                            ctypes.byref(got))
                assert rc == ps.PSB_OK, (op, call, rc)
                if op == ps.PS_SUM:
                    # the tolerance of the reduction tests
                    assert abs(got.value - want) <= 1e-13 * abssum, (call, got.value, want)
                else:
                    assert got.value == want, (op, call)
    finally:
        ps.PSGridFree(g)


@pytest.mark.gpu
def test_noalloc_rejects_extents_beyond_the_maximum():
    g = ps.grid_new(ps.PS_FLOAT, (8, 8, 8))
    try:
        origin, _, strides = _device_view(g)
        big = (ctypes.c_int64 * 3)(8, 8, 2147483648)
        got = ctypes.c_double()
        rc = lib.psb_reduce_noalloc(origin, ps.PS_FLOAT, ps.PS_SUM, big, strides, None,
                                    ctypes.byref(got))
        assert rc == ps.PSB_ERR_INVALID
    finally:
        ps.PSGridFree(g)
