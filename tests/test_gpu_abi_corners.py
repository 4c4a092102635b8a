"""Corners of the drop-in ABI, on the GPU, through the C entry points.

* Staggered grids in one map: examples/test_staggered_grid.c reads a grid of
  (N+1)^3 points at (x..x+1, y..y+1, z..z+1) and writes an N^3 grid over the
  domain [0, N)^3 (lines 6-14 and 24-27). Run here as a generic stencil and
  as a DSL stencil function, both against the oracle port and against the
  eight-point sum evaluated in float in the source's order.
* __PSGridSet / __PSGridGet (runtime/libphysis_rt_cuda.cc:164-179,
  include/physis/physis_ref.h:54-55): one element written or read at an
  index given as varargs, on dense (reference layout) and pitched grids of
  every element type, 1-D to 3-D; a periodic 7-point step after a set on a
  face point, which must see the new value through the wrapped halo.
"""
import ctypes

import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U

pytestmark = pytest.mark.gpu

STAGGERED_OFFSETS = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1),
                     (1, 1, 1)]

STAGGERED_DSL = """
void staggered_sum(const int x, const int y, const int z,
                   PSGrid3DFloat g1, PSGrid3DFloat g2) {
  float v = PSGridGet(g2, x, y, z) + PSGridGet(g2, x+1, y, z)
            + PSGridGet(g2, x, y+1, z) + PSGridGet(g2, x, y, z+1)
            + PSGridGet(g2, x+1, y+1, z) + PSGridGet(g2, x+1, y, z+1)
            + PSGridGet(g2, x, y+1, z+1) + PSGridGet(g2, x+1, y+1, z+1);
  PSGridEmit(g1, v);
}
"""


def _staggered_desc():
    xyz = (0, 1, 2)
    return dict(ndims=3, grids=[(ps.PS_FLOAT, xyz), (ps.PS_FLOAT, xyz)], out=0,
                accum=ps.PS_FLOAT, terms=[ps.get(1, o) for o in STAGGERED_OFFSETS])


def _staggered_host(g2, n):
    """The eight-point sum in float, left to right in the source's order."""
    acc = None
    for dx, dy, dz in STAGGERED_OFFSETS:
        v = g2[dz:dz + n[2], dy:dy + n[1], dx:dx + n[0]]
        acc = v.copy() if acc is None else (acc + v).astype(np.float32)
    return acc


def _run_staggered(kernel_id, n, layout, g2_host):
    g1 = ps.grid_new(ps.PS_FLOAT, n, layout)
    g2 = ps.grid_new(ps.PS_FLOAT, tuple(v + 1 for v in n), layout)
    try:
        ps.PSGridCopyin(g1, np.zeros(tuple(reversed(n)), np.float32))
        ps.PSGridCopyin(g2, g2_host)
        dom = ps.PSDomain3DNew(0, n[0], 0, n[1], 0, n[2])
        ps.PSStencilRun(ps.PSStencilMap(kernel_id, dom, g1, g2), 1)
        return ps.PSGridCopyout(g1)
    finally:
        ps.PSGridFree(g1)
        ps.PSGridFree(g2)


STAGGERED_SIZES = [(2, 2, 2), (33, 17, 9), (64, 40, 21)]


@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("n", STAGGERED_SIZES)
def test_staggered_generic_matches_oracle(n, layout):
    d = _staggered_desc()
    st = ps.GenericStencil(d["ndims"], d["grids"], d["out"], d["accum"], d["terms"])
    shape2 = tuple(v + 1 for v in reversed(n))
    # The reference's input is a ramp (indata[i] = i); random values too.
    for g2_host in (np.arange(np.prod(shape2), dtype=np.float32).reshape(shape2),
                    np.random.default_rng(5).random(shape2, dtype=np.float32)):
        got = _run_staggered(st.kernel_id, n, U.LAYOUTS[layout], g2_host)
        a1 = np.zeros(tuple(reversed(n)), np.float32)
        a2 = g2_host.copy()
        oracle.generic_apply(st.struct, [a1, a2], [0, 0, 0], list(n))
        assert U.bits_equal(got, a1)
        assert U.bits_equal(got, _staggered_host(g2_host, n))


def test_staggered_dsl_matches_oracle(tmp_path):
    from physis_b200 import dsl
    ps.PSInit()
    k = dsl.compile_stencils(STAGGERED_DSL, str(tmp_path))["staggered_sum"]
    for n in STAGGERED_SIZES:
        shape2 = tuple(v + 1 for v in reversed(n))
        g2_host = np.random.default_rng(6).random(shape2, dtype=np.float32)
        for layout in sorted(U.LAYOUTS):
            got = _run_staggered(k.kernel_id, n, U.LAYOUTS[layout], g2_host)
            assert U.bits_equal(got, _staggered_host(g2_host, n)), (n, layout)


def test_staggered_map_refuses_reads_past_the_larger_grid():
    """With both grids N^3 the (x+1) reads leave the grid: refused at map
    time instead of reading out of bounds."""
    d = _staggered_desc()
    st = ps.GenericStencil(d["ndims"], d["grids"], d["out"], d["accum"], d["terms"])
    g1 = ps.grid_new(ps.PS_FLOAT, (8, 8, 8))
    g2 = ps.grid_new(ps.PS_FLOAT, (8, 8, 8))
    try:
        with pytest.raises(ps.PhysisError):
            ps.PSStencilMap(st.kernel_id, ps.PSDomain3DNew(0, 8, 0, 8, 0, 8), g1, g2)
    finally:
        ps.PSGridFree(g1)
        ps.PSGridFree(g2)


# ---------------------------------------------------------------------------
# __PSGridSet / __PSGridGet
# ---------------------------------------------------------------------------
_set = getattr(ps.lib, "__PSGridSet")
_get = getattr(ps.lib, "__PSGridGet")
_set.restype = None
_get.restype = None


def _idx_args(idx):
    return [ctypes.c_int32(int(v)) for v in idx]


def grid_set(g, idx, value):
    buf = np.array([value], dtype=g.dtype)
    _set(g.ptr, ctypes.c_void_p(buf.ctypes.data), *_idx_args(idx))


def grid_get(g, idx):
    buf = np.zeros(1, dtype=g.dtype)
    _get(g.ptr, ctypes.c_void_p(buf.ctypes.data), *_idx_args(idx))
    return buf[0]


def _new(type_, dims, layout):
    if layout == ps.LAYOUT_DENSE:
        return ps.PSGridNewDense(type_, dims)
    return ps.grid_new(type_, dims, layout)


@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("type_", [ps.PS_FLOAT, ps.PS_DOUBLE, ps.PS_INT, ps.PS_LONG])
@pytest.mark.parametrize("dims", [(37,), (13, 9), (11, 7, 5)])
def test_set_get_round_trip(dims, type_, layout):
    ps.PSInit()
    g = _new(type_, dims, U.LAYOUTS[layout])
    try:
        dt = g.dtype
        shape = tuple(reversed(dims))
        rng = np.random.default_rng(len(dims) * 10 + type_)
        base = (rng.random(shape) * 1000).astype(dt)
        ps.PSGridCopyin(g, base)
        want = base.copy()
        # corners, faces and a few interior points
        pts = {tuple(0 for _ in dims), tuple(v - 1 for v in dims)}
        for _ in range(12):
            pts.add(tuple(int(rng.integers(0, v)) for v in dims))
        for k, p in enumerate(sorted(pts)):
            val = dt(-(k + 1) * 7)
            grid_set(g, p, val)
            want[tuple(reversed(p))] = val
        for p in sorted(pts):
            assert grid_get(g, p) == want[tuple(reversed(p))], p
        # untouched points keep their values: the whole grid equals the host copy
        assert U.bits_equal(ps.PSGridCopyout(g), want)
        # the last element of the grid (x fastest) is reachable
        last = tuple(v - 1 for v in dims)
        assert grid_get(g, last) == want[tuple(reversed(last))]
    finally:
        ps.PSGridFree(g)


@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
def test_periodic_step_after_set_sees_the_new_value(layout):
    """A periodic map reads wrapped neighbours; after __PSGridSet on face
    points the next step must read the new values there (the pitched
    layout's resident halo is refreshed)."""
    ps.PSInit()
    nx, ny, nz = 20, 12, 9
    f = np.random.default_rng(9).random((nz, ny, nx), dtype=np.float32)
    coef = [0.1, 0.1, 0.1, 0.1, 0.1, 0.1, 0.4]
    lay = U.LAYOUTS[layout]
    g1 = _new(ps.PS_FLOAT, (nx, ny, nz), lay)
    g2 = _new(ps.PS_FLOAT, (nx, ny, nz), lay)
    try:
        ps.PSGridCopyin(g1, f)
        dom = ps.PSDomain3DNew(0, nx, 0, ny, 0, nz)
        m1 = ps.PSStencilMap(ps.DIFFUSION7_PERIODIC, dom, g1, g2, *coef)
        m2 = ps.PSStencilMap(ps.DIFFUSION7_PERIODIC, dom, g2, g1, *coef)
        ps.PSStencilRun(m1, m2, 1)  # the halo of g1 is established and current
        host = oracle.diffusion7(f, 2, np.asarray(coef, np.float32), periodic=True)
        assert U.bits_equal(ps.PSGridCopyout(g1), host)
        for k, p in enumerate([(0, 3, 4), (nx - 1, 5, 2), (7, 0, 1), (2, ny - 1, 8), (4, 6, 0),
                               (9, 2, nz - 1), (0, 0, 0), (nx - 1, ny - 1, nz - 1)]):
            v = np.float32(5.0 + k)
            grid_set(g1, p, v)
            host[p[2], p[1], p[0]] = v
        ps.PSStencilRun(m1, m2, 1)
        want = oracle.diffusion7(host, 2, np.asarray(coef, np.float32), periodic=True)
        assert U.bits_equal(ps.PSGridCopyout(g1), want)
        assert grid_get(g1, (nx - 1, 0, 3)) == want[3, 0, nx - 1]
    finally:
        ps.PSGridFree(g1)
        ps.PSGridFree(g2)
