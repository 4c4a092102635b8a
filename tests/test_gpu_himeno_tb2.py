"""Himeno with two sweeps per pass (k_himeno_tb2): selected by a tune entry
with t_depth = 2, it must leave both pressure grids exactly as the
single-sweep run does (bit for bit against the oracle) and give every
sweep's residual within the tolerance of the single-sweep kernel's, for
ragged shapes (partial tiles in x, y and z), sub-chunk z extents, odd and
even pair counts, with and without residual histories."""
import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U

pytestmark = pytest.mark.gpu


def _tb2(dims, zc):
    ps.tune_set(ps.HIMENO19, ps.PS_FLOAT, dims, impl=ps.IMPL_TMA, tile_x=64, tile_y=8,
                z_chunk=zc, stages=6, t_depth=2)


@pytest.mark.parametrize("shape,zc", [((9, 9, 9), 16), ((35, 33, 65), 16), ((70, 20, 130), 32),
                                      ((40, 17, 257), 64), ((129, 67, 66), 16),
                                      ((6, 70, 6), 16)])
@pytest.mark.parametrize("sweeps", [6, 8, 14])
def test_two_sweep_pass_bit_exact(shape, zc, sweeps):
    ps.PSInit()
    nz, ny, nx = shape
    p, coef = U.himeno_inputs(shape, 3)
    _tb2((nx, ny, nz), zc)
    try:
        got, gosa = U.himeno_gpu(p, coef, 0.8, sweeps)
        got_nr, _ = U.himeno_gpu(p, coef, 0.8, sweeps, residual=False)
    finally:
        ps.tune_set(ps.HIMENO19, ps.PS_FLOAT, (nx, ny, nz), impl=ps.IMPL_TMA, tile_x=64,
                    tile_y=8, z_chunk=16, stages=6, t_depth=1)
    want, wgosa = oracle.himeno(p, coef, 0.8, sweeps)
    assert U.bits_equal(got, want)
    assert U.bits_equal(got_nr, want)
    assert np.allclose(gosa, wgosa, rtol=1e-12, atol=0)


def test_both_grids_end_as_in_the_single_sweep_run():
    """After PSStencilRun(m1, m2, n) p0 holds sweep 2n and p1 sweep 2n-1,
    whichever kernel ran."""
    ps.PSInit()
    shape = (33, 40, 70)
    nz, ny, nx = shape
    dims = (nx, ny, nz)
    p, coef = U.himeno_inputs(shape, 4)
    _tb2(dims, 16)
    gs = [ps.grid_new(ps.PS_FLOAT, dims) for _ in range(14)]
    try:
        ps.PSGridCopyin(gs[0], p)
        ps.PSGridCopyin(gs[1], p)
        for i in range(12):
            ps.PSGridCopyin(gs[2 + i], coef[i])
        d = ps.PSDomain3DNew(1, nx - 1, 1, ny - 1, 1, nz - 1)
        m1 = ps.PSStencilMap(ps.HIMENO19, d, *([gs[0], gs[1]] + gs[2:]), 0.8)
        m2 = ps.PSStencilMap(ps.HIMENO19, d, *([gs[1], gs[0]] + gs[2:]), 0.8)
        ps.PSStencilRun(m1, m2, 7)
        launches = ps.last_run_stats()[1]
        a, b = ps.PSGridCopyout(gs[0]), ps.PSGridCopyout(gs[1])
    finally:
        ps.tune_set(ps.HIMENO19, ps.PS_FLOAT, dims, impl=ps.IMPL_TMA, tile_x=64, tile_y=8,
                    z_chunk=16, stages=6, t_depth=1)
        for g in gs:
            ps.PSGridFree(g)
    assert U.bits_equal(a, oracle.himeno(p, coef, 0.8, 14)[0])
    assert U.bits_equal(b, oracle.himeno(p, coef, 0.8, 13)[0])
    assert launches < 14  # fused launches ran (6 two-sweep passes + 2 single sweeps)
