"""Himeno 19-point Jacobi against the oracle: pressure bit for bit, the
fused FP64 residual within 1e-12 relative (only the summation order
differs)."""
import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U

IMPLS = {"plain": ps.IMPL_PLAIN, "tma": ps.IMPL_TMA}


@pytest.mark.gpu
@pytest.mark.parametrize("impl", sorted(IMPLS))
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("shape", [(3, 3, 3), (6, 7, 9), (17, 12, 19), (33, 33, 65), (20, 9, 130)])
def test_himeno_bit_exact(shape, layout, impl):
    p, coef = U.himeno_inputs(shape, 11)
    want, gosa = oracle.himeno(p, coef, 0.8, 4)
    got, g = U.himeno_gpu(p, coef, 0.8, 4, impl=IMPLS[impl], layout=U.LAYOUTS[layout])
    assert U.bits_equal(got, want)
    assert np.allclose(g, gosa, rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_himeno_c3_size_two_sweeps():
    """257 x 257 x 513 (the C3 grid), two sweeps, TMA path."""
    p, coef = U.himeno_inputs((513, 257, 257), 12)
    want, gosa = oracle.himeno(p, coef, 0.8, 2)
    got, g = U.himeno_gpu(p, coef, 0.8, 2, impl=ps.IMPL_TMA)
    assert U.bits_equal(got, want)
    assert np.allclose(g, gosa, rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_himeno_residual_deterministic():
    p, coef = U.himeno_inputs((65, 65, 129), 13)
    _, g1 = U.himeno_gpu(p, coef, 0.8, 6)
    _, g2 = U.himeno_gpu(p, coef, 0.8, 6)
    assert g1 == g2
