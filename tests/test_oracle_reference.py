"""The oracle port against the reference CPU target itself (CPU only).

libphysis_rt_ref is compiled from the reference's runtime sources
(oracle/Makefile `ref`); the translator-shaped programs in oracle/ref_paths.c
drive it like generated code would. The port must agree bit for bit on the
benchmark stencils (7-point diffusion clamped/periodic in float and double,
Himeno) and on PSReduce's sequential fold.
"""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.skipif(not oracle.ref_available(),
                                reason="reference runtime not built (no reference sources)")

COEF = [0.1, 0.1, 0.1, 0.1, 0.1, 0.1, 0.4]


def _field(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    return rng.random(shape).astype(dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("shape", [(8, 9, 10), (17, 5, 33), (3, 3, 3)])
def test_diffusion_port_equals_reference(dtype, periodic, shape):
    f = _field(shape, dtype, 1)
    ref, _ = oracle.ref_diffusion7(f, 6, np.asarray(COEF, dtype), periodic)
    port = oracle.diffusion7(f, 6, np.asarray(COEF, dtype), periodic)
    assert np.array_equal(ref.view(np.uint8), port.view(np.uint8))


def _himeno_inputs(shape, seed):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    u = lambda lo, hi: (lo + (hi - lo) * rng.random(shape)).astype(np.float32)
    a = [u(0.9, 1.1) for _ in range(3)] + [(u(0.95, 1.05) / np.float32(6)).astype(np.float32)]
    b = [u(-0.01, 0.01) for _ in range(3)]
    c = [u(0.9, 1.1) for _ in range(3)]
    bnd = np.ones(shape, np.float32)
    bnd[0, :, :] = bnd[-1, :, :] = bnd[:, 0, :] = bnd[:, -1, :] = bnd[:, :, 0] = bnd[:, :, -1] = 0
    wrk1 = np.zeros(shape, np.float32)
    k = np.arange(nz, dtype=np.float32)
    p = np.broadcast_to(((k * k) / np.float32((nz - 1) * (nz - 1)))[:, None, None],
                        shape).astype(np.float32)
    return p, a + b + c + [bnd, wrk1]


@pytest.mark.parametrize("shape", [(9, 7, 6), (17, 12, 19)])
def test_himeno_port_equals_reference(shape):
    p, coef = _himeno_inputs(shape, 3)
    ref, _ = oracle.ref_himeno(p, coef, 0.8, 4)
    port, gosa = oracle.himeno(p, coef, 0.8, 4)
    assert np.array_equal(ref.view(np.uint32), port.view(np.uint32))
    assert len(gosa) == 4 and np.all(np.isfinite(gosa))


@pytest.mark.parametrize("op", [oracle.PS_MAX, oracle.PS_MIN, oracle.PS_SUM, oracle.PS_PROD])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_reduce_fold_equals_reference(op, dtype):
    rng = np.random.default_rng(7)
    d = (0.5 + rng.random(4099)).astype(dtype)
    assert oracle.ref_reduce(op, d) == oracle.fold(op, d)
