"""7-point diffusion kernels (plain and TMA) against the oracle, bit for bit.

Ragged and odd extents exercise partial tiles, both grid layouts, float and
double, clamped and periodic faces, sub-domains, and the C2 sizes (512^3
float, 256^3 double) for two steps against the single-threaded oracle.
"""
import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U

COEF = [0.1, 0.1, 0.1, 0.1, 0.1, 0.1, 0.4]
IMPLS = {"plain": ps.IMPL_PLAIN, "tma": ps.IMPL_TMA}
SHAPES = [(1, 1, 1), (2, 3, 5), (3, 1, 33), (8, 8, 8), (5, 7, 31), (17, 3, 33), (9, 4, 257),
          (33, 40, 64)]


def _field(shape, dtype, seed=0):
    return np.random.default_rng(seed).random(shape).astype(dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("impl", sorted(IMPLS))
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", SHAPES)
def test_clamped_bit_exact(shape, dtype, layout, impl):
    f = _field(shape, dtype, 1)
    coef = np.asarray(COEF, dtype)
    want = oracle.diffusion7(f, 4, coef)
    got = U.diffusion_gpu(f, 4, [float(c) for c in coef], impl=IMPLS[impl],
                          layout=U.LAYOUTS[layout])
    assert U.bits_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("impl", sorted(IMPLS))
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(2, 3, 4), (8, 8, 8), (5, 7, 31), (17, 3, 33), (12, 10, 72)])
def test_periodic_bit_exact(shape, dtype, layout, impl):
    f = _field(shape, dtype, 2)
    coef = np.asarray(COEF, dtype)
    want = oracle.diffusion7(f, 6, coef, periodic=True)
    got = U.diffusion_gpu(f, 6, [float(c) for c in coef], periodic=True, impl=IMPLS[impl],
                          layout=U.LAYOUTS[layout])
    assert U.bits_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("impl", sorted(IMPLS))
@pytest.mark.parametrize("dom", [((1, 1, 1), (31, 15, 9)), ((3, 0, 2), (30, 16, 10)),
                                 ((0, 5, 0), (5, 6, 10))])
def test_subdomain_bit_exact(dom, impl):
    shape = (10, 16, 32)
    f = _field(shape, np.float32, 3)
    coef = np.asarray(COEF, np.float32)
    want = oracle.diffusion7(f, 4, coef, lo=dom[0], hi=dom[1])
    got = U.diffusion_gpu(f, 4, [float(c) for c in coef], impl=IMPLS[impl], dom=dom)
    assert U.bits_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_odd_step_counts_and_graph_replay(graph):
    f = _field((16, 16, 40), np.float32, 4)
    coef = np.asarray(COEF, np.float32)
    for steps in (1, 3, 34, 70):
        want = oracle.diffusion7(f, steps, coef)
        got = U.diffusion_gpu(f, steps, [float(c) for c in coef], graph=graph)
        assert U.bits_equal(got, want), steps


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,n", [(np.float32, 512), (np.float64, 256)])
def test_full_size_two_steps(dtype, n):
    """The C2 workloads: two steps at full size, TMA path, against the oracle."""
    shape = (n, n, n)
    rng = np.random.default_rng(5)
    f = rng.random(shape, dtype=np.float32).astype(dtype)
    coef = np.asarray(COEF, dtype)
    want = oracle.diffusion7(f, 2, coef)
    got = U.diffusion_gpu(f, 2, [float(c) for c in coef], impl=ps.IMPL_TMA)
    assert U.bits_equal(got, want)


@pytest.mark.gpu
def test_tma_equals_plain_many_steps():
    """Size-independent property at 512^3: the TMA and plain kernels agree
    bit for bit after 20 steps."""
    f = np.random.default_rng(6).random((512, 512, 512), dtype=np.float32)
    a = U.diffusion_gpu(f, 20, COEF, impl=ps.IMPL_TMA)
    b = U.diffusion_gpu(f, 20, COEF, impl=ps.IMPL_PLAIN)
    assert U.bits_equal(a, b)


@pytest.mark.gpu
def test_periodic_conserves_total():
    """With coefficients summing to 1 the periodic update conserves the
    total up to rounding: |sum_after - sum_before| <= 1e-5 relative."""
    f = np.random.default_rng(8).random((128, 96, 160)).astype(np.float64)
    out = U.diffusion_gpu(f, 10, COEF, periodic=True, impl=ps.IMPL_TMA)
    assert abs(out.sum() - f.sum()) <= 1e-12 * f.size


def _tb_run(field, pairs, zchunk):
    """PSStencilRun(m(g1->g2), m(g2->g1), pairs) with two-step temporal
    blocking selected for this grid size; returns (g1, g2)."""
    nz, ny, nx = field.shape
    dims = (nx, ny, nz)
    old = ps.tune_get(ps.DIFFUSION7, ps.PS_FLOAT, dims)
    ps.tune_set(ps.DIFFUSION7, ps.PS_FLOAT, dims, impl=ps.IMPL_TMA, tile_x=128, tile_y=8,
                z_chunk=zchunk, stages=6, t_depth=2)
    g1 = ps.grid_new(ps.PS_FLOAT, dims)
    g2 = ps.grid_new(ps.PS_FLOAT, dims)
    try:
        ps.PSGridCopyin(g1, field)
        d = ps.PSDomain3DNew(0, nx, 0, ny, 0, nz)
        m1 = ps.PSStencilMap(ps.DIFFUSION7, d, g1, g2, *COEF)
        m2 = ps.PSStencilMap(ps.DIFFUSION7, d, g2, g1, *COEF)
        ps.PSStencilRun(m1, m2, pairs)
        return ps.PSGridCopyout(g1), ps.PSGridCopyout(g2), ps.last_run_stats()[1]
    finally:
        ps.PSGridFree(g1)
        ps.PSGridFree(g2)
        ps.tune_set(ps.DIFFUSION7, ps.PS_FLOAT, dims, **old)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,pairs,zchunk", [
    ((8, 16, 128), 3, 8),        # one tile exactly
    ((37, 50, 130), 5, 16),      # ragged tiles in x and y
    ((40, 64, 256), 4, 12),      # several tiles, partial z chunk
    ((9, 33, 200), 1, 4),        # one pair only: no two-step launch
    ((70, 20, 300), 6, 32),
])
def test_temporal_blocking_bit_exact(shape, pairs, zchunk):
    """Two steps per launch give the same bits as single steps, in both grids
    (g1 after 2*pairs steps, g2 after 2*pairs - 1)."""
    f = np.random.default_rng(sum(shape)).random(shape, dtype=np.float32)
    got1, got2, launches = _tb_run(f, pairs, zchunk)
    want2 = oracle.diffusion7(f, 2 * pairs - 1, COEF)
    want1 = oracle.diffusion7(want2, 1, COEF)
    assert U.bits_equal(got1, want1)
    assert U.bits_equal(got2, want2)
    fused = (pairs - 1) & ~1
    assert launches == fused + 2 * (pairs - fused)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,pairs,zchunk", [
    ((8, 16, 128), 3, 8),
    ((37, 50, 130), 5, 16),
    ((70, 20, 300), 6, 32),
])
def test_temporal_blocking_fma_mode_equals_single_fma_steps(shape, pairs, zchunk):
    """In the FMA arithmetic mode the two-step kernel computes every point as
    the single-step FMA kernel does: the same bits as single FMA steps."""
    f = np.random.default_rng(7 + sum(shape)).random(shape, dtype=np.float32)
    nz, ny, nx = shape
    dims = (nx, ny, nz)
    old = ps.tune_get(ps.DIFFUSION7, ps.PS_FLOAT, dims)
    ps.set_fp_mode(ps.FP_FMA)
    try:
        got1, got2, launches = _tb_run(f, pairs, zchunk)
        ps.tune_set(ps.DIFFUSION7, ps.PS_FLOAT, dims, impl=ps.IMPL_TMA, tile_x=128, tile_y=8,
                    z_chunk=zchunk, stages=6, t_depth=1)
        g1 = ps.grid_new(ps.PS_FLOAT, dims)
        g2 = ps.grid_new(ps.PS_FLOAT, dims)
        try:
            ps.PSGridCopyin(g1, f)
            d = ps.PSDomain3DNew(0, nx, 0, ny, 0, nz)
            m1 = ps.PSStencilMap(ps.DIFFUSION7, d, g1, g2, *COEF)
            m2 = ps.PSStencilMap(ps.DIFFUSION7, d, g2, g1, *COEF)
            ps.PSStencilRun(m1, m2, pairs)
            want1, want2 = ps.PSGridCopyout(g1), ps.PSGridCopyout(g2)
        finally:
            ps.PSGridFree(g1)
            ps.PSGridFree(g2)
    finally:
        ps.set_fp_mode(ps.FP_EXACT)
        ps.tune_set(ps.DIFFUSION7, ps.PS_FLOAT, dims, **old)
    fused = (pairs - 1) & ~1
    assert launches == fused + 2 * (pairs - fused)
    assert U.bits_equal(got1, want1)
    assert U.bits_equal(got2, want2)
    # and not the exact arithmetic's bits (the FMA form ran)
    assert not U.bits_equal(got1, oracle.diffusion7(f, 2 * pairs, COEF))
