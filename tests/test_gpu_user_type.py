"""Grids of user-defined point types (DeclareGrid3D with struct members):
a host array of records on the host, one pitched device grid per scalar
component. After test_user-defined-type-copyin-copyout.c and
test_user-defined-type-kernel-copy.c of the reference's system tests, plus
a struct of mixed member types read by a stencil."""
import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U

pytestmark = pytest.mark.gpu

N = 32
POINT = np.dtype([("p", np.float32, (2, 3))])  # struct Point { float p[2][3]; }


def _point_grid(dims):
    return ps.grid_new_user(dims, [(ps.PS_FLOAT, 6, 0)], POINT.itemsize)


def _ramp(dims):
    n = int(np.prod(dims))
    a = np.zeros(tuple(reversed(dims)), POINT)
    a["p"] = (1.0 + np.arange(n * 6, dtype=np.float32)).reshape(a.shape + (2, 3))
    return a


def test_copyin_copyout_round_trip():
    dims = (N, N, N)
    g = _point_grid(dims)
    try:
        a = _ramp(dims)
        ps.user_copyin(g, a)
        out = np.zeros_like(a)
        ps.user_copyout(g, out)
        assert np.array_equal(out["p"], a["p"])
        # Each component holds its scalar of every record, in the grid's shape.
        c4 = ps.PSGridCopyout(ps.component(g, 0, 4))
        assert np.array_equal(c4, a["p"][..., 1, 1])
    finally:
        ps.PSGridFree(g)


def test_kernel_copy_per_component():
    """copy(x,y,z,g1,g2): g2.p[i][j] = g1(x,y,z).p[i][j], as one map per
    component run together."""
    dims = (N, N, N)
    g1, g2 = _point_grid(dims), _point_grid(dims)
    try:
        a = _ramp(dims)
        ps.user_copyin(g1, a)
        init = np.zeros_like(a)
        init["p"] = -1
        ps.user_copyin(g2, init)
        st = ps.GenericStencil(3, [(ps.PS_FLOAT, (0, 1, 2))] * 2, 1, ps.PS_FLOAT,
                               [ps.get(0, (0, 0, 0))])
        dom = ps.PSDomain3DNew(0, N, 0, N, 0, N)
        maps = [ps.PSStencilMap(st.kernel_id, dom, ps.component(g1, 0, k), ps.component(g2, 0, k))
                for k in range(6)]
        ps.PSStencilRun(*maps)
        out = np.zeros_like(a)
        ps.user_copyout(g2, out)
        assert np.array_equal(out["p"], a["p"])
    finally:
        ps.PSGridFree(g1)
        ps.PSGridFree(g2)


MIX = np.dtype([("a", np.float32), ("b", np.float64, (2,)), ("c", np.int32), ("d", np.int64)],
               align=True)


def test_mixed_struct_and_stencil_on_components():
    dims = (19, 7, 11)
    fields = [(ps.PS_FLOAT, 1, MIX.fields["a"][1]), (ps.PS_DOUBLE, 2, MIX.fields["b"][1]),
              (ps.PS_INT, 1, MIX.fields["c"][1]), (ps.PS_LONG, 1, MIX.fields["d"][1])]
    g = ps.grid_new_user(dims, fields, MIX.itemsize)
    h = ps.grid_new(ps.PS_FLOAT, dims)
    try:
        rng = np.random.default_rng(3)
        a = np.zeros(tuple(reversed(dims)), MIX)
        a["a"] = rng.random(a.shape, dtype=np.float32)
        a["b"] = rng.random(a.shape + (2,))
        a["c"] = rng.integers(-1000, 1000, a.shape)
        a["d"] = rng.integers(-2 ** 40, 2 ** 40, a.shape)
        ps.user_copyin(g, a)
        out = np.zeros_like(a)
        ps.user_copyout(g, out)
        for f in ("a", "b", "c", "d"):
            assert np.array_equal(out[f], a[f]), f
        # A 7-point stencil over component a (clamped), written to h.
        coef = [0.1, 0.1, 0.1, 0.1, 0.1, 0.1, 0.4]
        m = ps.PSStencilMap(ps.DIFFUSION7, ps.PSDomain3DNew(0, dims[0], 0, dims[1], 0, dims[2]),
                            ps.component(g, 0), h, *coef)
        ps.PSStencilRun(m)
        want = oracle.diffusion7(np.ascontiguousarray(a["a"]), 1, coef)
        assert U.bits_equal(ps.PSGridCopyout(h), want)
    finally:
        ps.PSGridFree(g)
        ps.PSGridFree(h)


def test_invalid_types_are_refused():
    with pytest.raises(ps.PhysisError):
        ps.grid_new_user((4, 4, 4), [(ps.PS_DOUBLE, 1, 4)], 16)  # misaligned double
    with pytest.raises(ps.PhysisError):
        ps.grid_new_user((4, 4, 4), [(ps.PS_FLOAT, 5, 0)], 16)   # field past the record


def test_whole_point_grid_is_refused_where_it_has_no_storage():
    """A point-type grid keeps its data in its components: calls that would
    touch the grid's own storage (fill, reduce, built-in or generic maps,
    grid copy) refuse it up front, before any device work."""
    dims = (8, 8, 8)
    g, h = _point_grid(dims), _point_grid(dims)
    f = ps.grid_new(ps.PS_FLOAT, dims)
    try:
        codes = []
        codes.append(ps.lib.psb_grid_fill(g.ptr, ps.FILL_CONST, 0, 1.0, 1.0))
        codes.append(ps.lib.psb_grid_copy(g.ptr, h.ptr))
        dom = ps.PSDomain3DNew(1, 7, 1, 7, 1, 7)
        for k, gs in ((ps.DIFFUSION7, [g, f]), (ps.DIFFUSION7, [f, g])):
            with pytest.raises(ps.PhysisError) as e:
                ps.PSStencilMap(k, dom, *gs, *([0.1] * 7))
            codes.append(e.value.status)
        st = ps.GenericStencil(3, [(ps.PS_FLOAT, (0, 1, 2))] * 2, 1, ps.PS_FLOAT,
                               [ps.get(0, (0, 0, 0))])
        with pytest.raises(ps.PhysisError) as e:
            ps.PSStencilMap(st.kernel_id, dom, g, f)
        codes.append(e.value.status)
        with pytest.raises(ps.PhysisError) as e:
            ps.PSReduce(ps.PS_SUM, g)
        codes.append(e.value.status)
        assert codes == [ps.PSB_ERR_INVALID] * len(codes)
        ps.sync()
    finally:
        for x in (g, h, f):
            ps.PSGridFree(x)
