"""PSReduce against the reference's fold and an FP64 oracle.

MAX/MIN are exact. SUM accumulates in FP64 (Neumaier for double grids):
it must equal the compensated FP64 sum within 1e-13 relative, and the
reference's sequential float fold within its error bound gamma_n*sum|x|.
"""
import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U


def _grid(a, layout):
    t = ps.PS_FLOAT if a.dtype == np.float32 else ps.PS_DOUBLE
    g = ps.grid_new(t, tuple(reversed(a.shape)), layout)
    ps.PSGridCopyin(g, a)
    return g


SHAPES = [(1, 1, 1), (1, 1, 7), (3, 5, 31), (17, 33, 65), (64, 64, 64), (5, 300, 257)]


@pytest.mark.gpu
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", SHAPES)
def test_reduce_ops(shape, dtype, layout):
    rng = np.random.default_rng(21)
    a = (rng.random(shape) - 0.3).astype(dtype)
    g = _grid(a, U.LAYOUTS[layout])
    try:
        assert ps.PSReduce(ps.PS_MAX, g) == a.max()
        assert ps.PSReduce(ps.PS_MIN, g) == a.min()
        s64, abss = oracle.sum_f64(a)
        got = ps.reduce64(ps.PS_SUM, g)
        assert abs(got - s64) <= 1e-13 * abss + 1e-300
        fold = float(oracle.fold(ps.PS_SUM, a))
        n = a.size
        u = 2.0 ** -24 if dtype == np.float32 else 2.0 ** -53
        gamma = n * u / (1 - n * u)
        assert abs(ps.PSReduce(ps.PS_SUM, g) - fold) <= gamma * abss + 4 * u * abs(fold)
        b = (0.999 + 0.002 * rng.random(shape)).astype(dtype)
        ps.PSGridCopyin(g, b)
        prod64 = float(np.prod(b.astype(np.float64)))
        assert abs(ps.reduce64(ps.PS_PROD, g) - prod64) <= 1e-12 * abs(prod64)
    finally:
        ps.PSGridFree(g)


@pytest.mark.gpu
def test_reduce_c1_style_sum_after_run():
    """C1's tail: PSReduce(&v, PS_SUM, g) of a diffused field, against the
    reference's own fold within its bound."""
    f = np.random.default_rng(22).random((64, 64, 64), dtype=np.float32)
    out = U.diffusion_gpu(f, 100, [0.1] * 6 + [0.4])
    g = _grid(out, ps.LAYOUT_PITCHED)
    try:
        v = ps.PSReduce(ps.PS_SUM, g)
        s64, abss = oracle.sum_f64(out)
        assert v == np.float32(s64)
        fold = float(oracle.fold(ps.PS_SUM, out))
        assert abs(v - fold) <= out.size * 2.0 ** -24 * abss
    finally:
        ps.PSGridFree(g)


@pytest.mark.gpu
def test_reduce_deterministic_and_subdomain():
    a = np.random.default_rng(23).random((40, 50, 60))
    g = _grid(a, ps.LAYOUT_PITCHED)
    try:
        r = [ps.reduce64(ps.PS_SUM, g) for _ in range(3)]
        assert r[0] == r[1] == r[2]
        d = ps.PSDomain3DNew(3, 50, 4, 40, 5, 30)
        sub = a[5:30, 4:40, 3:50]
        s64, abss = oracle.sum_f64(sub)
        assert abs(ps.reduce64(ps.PS_SUM, g, d) - s64) <= 1e-13 * abss
        assert ps.reduce64(ps.PS_MAX, g, d) == sub.max()
    finally:
        ps.PSGridFree(g)
