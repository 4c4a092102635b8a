"""psb_reduce_noalloc: the allocation-free reduction entry point.

Some callers may not call cudaMalloc: a host framework that owns all device
memory through its own allocator and counts it against a budget, or a
latency-critical loop in which an allocation would synchronise the device.
This entry point serves them by keeping its scratch in a fixed static device
array instead of allocating. Its results are checked here directly against
the oracle (compensated FP64 sum, exact maximum and minimum, sequential FP64
product) and against the allocating entry point, on two calls in a row,
for every element type, on a caller-created stream, and on padded and
sub-box views. Its argument checks run on the host.

This file is collected last on purpose, so a run that stops at the first
failure has already run every other test; it also passes alone in a fresh
process (it sets up its own grids).
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

# Tolerance of the reduction tests: SUM within 1e-13 relative to sum |x|.
SUM_RTOL = 1e-13


def _noalloc(origin, type_, op, ext, strides, stream=None):
    got = ctypes.c_double()
    e = (ctypes.c_int64 * 3)(*ext)
    s = (ctypes.c_int64 * 2)(*strides)
    rc = lib.psb_reduce_noalloc(ctypes.c_void_p(origin), type_, op, e, s, stream,
                                ctypes.byref(got))
    return rc, got.value


def _view(g, lo=(0, 0, 0), ext=None):
    """Device address of element lo of a grid, the extents from there and
    the grid's strides (elements)."""
    origin = ps.PSGridStruct.from_address(g.ptr.value).p0
    lay = g.layout()
    esize = np.dtype(g.dtype).itemsize
    addr = origin + esize * (lo[0] + lo[1] * lay["stride_y"] + lo[2] * lay["stride_z"])
    ext = ext or tuple(n - l for n, l in zip(g.dims, lo))
    return addr, ext, (lay["stride_y"], lay["stride_z"])


def _want(op, a):
    """Oracle value of op over a (float, double or integer array) in FP64."""
    if op == ps.PS_SUM:
        if a.dtype.kind == "f":
            return oracle.sum_f64(a)
        return float(int(a.astype(np.int64).sum())), float(np.abs(a.astype(np.int64)).sum())
    if op == ps.PS_PROD:
        return oracle.fold(ps.PS_PROD, a.astype(np.float64)), None
    return float(a.max() if op == ps.PS_MAX else a.min()), None


def _check(op, got, want, abssum, exact):
    if op == ps.PS_SUM and not exact:
        assert abs(got - want) <= SUM_RTOL * abssum, (got, want)
    elif op == ps.PS_PROD and not exact:
        # FP64 products in another order: n roundings of 2^-53 at most
        assert abs(got - want) <= 1e-10 * abs(want), (got, want)
    else:
        assert got == want, (op, got, want)


def _data(dtype, shape, seed, op=None):
    rng = np.random.default_rng(seed)
    if op == ps.PS_PROD:
        if np.dtype(dtype).kind == "f":
            return (0.999 + 0.002 * rng.random(shape)).astype(dtype)
        a = np.where(rng.random(shape) < 0.5, -1, 1).astype(dtype)
        a.flat[rng.choice(a.size, 10, replace=False)] = 2
        return a
    if np.dtype(dtype).kind == "f":
        return (rng.random(shape) - 0.25).astype(dtype)
    return rng.integers(-1000, 1000, size=shape).astype(dtype)


TYPES = [(ps.PS_FLOAT, np.float32), (ps.PS_DOUBLE, np.float64), (ps.PS_INT, np.int32),
         (ps.PS_LONG, np.int64)]
OPS = [ps.PS_SUM, ps.PS_MAX, ps.PS_MIN, ps.PS_PROD]


@pytest.mark.gpu
@pytest.mark.parametrize("type_,dtype", TYPES)
def test_noalloc_matches_oracle_and_allocating_entry_point(type_, dtype):
    ps.PSInit()
    dims = (131, 45, 37)
    g = ps.grid_new(type_, dims)
    try:
        for op in OPS:
            a = _data(dtype, tuple(reversed(dims)), 41 + op, op)
            ps.PSGridCopyin(g, a)
            ps.sync()  # the copy-in ran on the runtime's stream
            want, abssum = _want(op, a)
            exact = np.dtype(dtype).kind == "i"
            alloc = ps.reduce64(op, g)
            origin, ext, strides = _view(g)
            for call in range(2):  # two calls in a row share the static scratch
                rc, got = _noalloc(origin, type_, op, ext, strides)
                assert rc == ps.PSB_OK, (op, call, rc)
                _check(op, got, want, abssum, exact)
                _check(op, got, alloc, abssum, exact)
    finally:
        ps.PSGridFree(g)


@pytest.mark.gpu
def test_noalloc_on_a_caller_stream_and_sub_box_views():
    """A stream the caller created (ordered after the copy-in by psb_sync),
    a sub-box of a pitched grid (strides larger than the extents, origin
    inside the grid) and a dense grid (strides equal to the extents)."""
    import torch
    ps.PSInit()
    dims = (200, 33, 19)
    a = _data(np.float32, tuple(reversed(dims)), 7)
    g = ps.grid_new(ps.PS_FLOAT, dims)
    gd = ps.PSGridNewDense(ps.PS_FLOAT, dims)
    stream = torch.cuda.Stream()
    try:
        ps.PSGridCopyin(g, a)
        ps.PSGridCopyin(gd, a)
        ps.sync()
        lo, ext = (3, 2, 1), (150, 30, 17)
        sub = a[lo[2]:lo[2] + ext[2], lo[1]:lo[1] + ext[1], lo[0]:lo[0] + ext[0]]
        views = [(_view(g, lo, ext), sub), (_view(g), a), (_view(gd), a)]
        gd_origin = ps.PSGridStruct.from_address(gd.ptr.value).p0
        assert views[2][0][2] == (dims[0], dims[0] * dims[1])
        assert views[2][0][0] == gd_origin
        for (origin, e, strides), host in views:
            for op in OPS:
                want, abssum = _want(op, host)
                for call in range(2):
                    rc, got = _noalloc(origin, ps.PS_FLOAT, op, e, strides,
                                       ctypes.c_void_p(stream.cuda_stream))
                    assert rc == ps.PSB_OK
                    _check(op, got, want, abssum, False)
        stream.synchronize()
    finally:
        ps.PSGridFree(g)
        ps.PSGridFree(gd)


@pytest.mark.gpu
def test_noalloc_rejects_extents_beyond_the_maximum():
    ps.PSInit()
    g = ps.grid_new(ps.PS_FLOAT, (8, 8, 8))
    try:
        origin, _, strides = _view(g)
        rc, _ = _noalloc(origin, ps.PS_FLOAT, ps.PS_SUM, (8, 8, 2147483648), strides)
        assert rc == ps.PSB_ERR_INVALID
    finally:
        ps.PSGridFree(g)


# Host-side argument checks. Every one of these is refused before the entry
# point touches the device, so the pointer below is never dereferenced and
# the tests run without a GPU.
FAKE = 1 << 20


@pytest.mark.parametrize("ext,strides", [
    ((8, 8, 2147483648), (8, 64)),             # nz beyond PSB_NOALLOC_MAX_EXTENT
    ((2147483648, 1, 1), (2147483648, 2147483648)),
    ((0, 8, 8), (8, 64)),                      # empty extent
    ((8, 8, 8), (7, 64)),                      # rows overlap
    ((8, 8, 8), (8, 63)),                      # planes overlap
    ((8, 8, 8), (2 ** 62, 2 ** 62)),           # plane stride below row stride x ny
    ((8, 8, 8), (8, 2 ** 62)),                 # last element beyond INT64_MAX / 8
    ((2147483647, 2147483647, 2), (2147483647, 2 ** 62)),
])
def test_noalloc_rejects_bad_views_on_the_host(ext, strides):
    rc, _ = _noalloc(FAKE, ps.PS_FLOAT, ps.PS_SUM, ext, strides)
    assert rc == ps.PSB_ERR_INVALID


@pytest.mark.parametrize("type_,op", [(7, ps.PS_SUM), (ps.PS_FLOAT, 9), (ps.PS_FLOAT, -1)])
def test_noalloc_rejects_bad_type_or_op_on_the_host(type_, op):
    rc, _ = _noalloc(FAKE, type_, op, (8, 8, 8), (8, 64))
    assert rc == ps.PSB_ERR_INVALID
