"""The contracted (FMA) arithmetic (PSB_FP_FMA) of the 7-point TMA kernels
and of generic tables compiled at run time (bound stated at the end).

Not bit-identical to the reference by design: the reference's term order
with one rounding per term instead of two. The stated tolerance is 4 ulp
per step: every point of one step, from the same input, lies within 4 ulp
(of the element type, at the exact value) of the exact value of the step,
which is computed here in extended precision from the same inputs and
coefficients (the reference's own rounded result is held to the same bar).
Over many steps the bound accumulates: after n steps the error against the
FP64 oracle stays within 4 n ulp."""
import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U

pytestmark = pytest.mark.gpu

COEF = [0.1, 0.1, 0.1, 0.1, 0.1, 0.1, 0.4]
ULP_PER_STEP = 4


def _ulp_err(got, exact):
    """Largest |got - exact| in ulp of got's type at the exact value."""
    dt = got.dtype
    e = np.asarray(exact, dtype=np.longdouble)
    ulp = np.spacing(np.abs(e).astype(dt)).astype(np.longdouble)
    return float(np.max(np.abs(got.astype(np.longdouble) - e) / ulp))


def _exact_step(f, periodic):
    """One 7-point step in extended precision (64-bit significand) from the
    same inputs and the coefficients rounded to the field's type."""
    c = [np.longdouble(np.asarray(v, dtype=f.dtype)) for v in COEF]
    ce, cw, cn, cs, ct, cb, cc = c
    u = f.astype(np.longdouble)
    if periodic:
        sh = lambda a, k, ax: np.roll(a, k, axis=ax)
        w, e = sh(u, 1, 2), sh(u, -1, 2)
        n, s = sh(u, 1, 1), sh(u, -1, 1)
        b, t = sh(u, 1, 0), sh(u, -1, 0)
    else:
        w = np.concatenate([u[:, :, :1], u[:, :, :-1]], 2)
        e = np.concatenate([u[:, :, 1:], u[:, :, -1:]], 2)
        n = np.concatenate([u[:, :1], u[:, :-1]], 1)
        s = np.concatenate([u[:, 1:], u[:, -1:]], 1)
        b = np.concatenate([u[:1], u[:-1]], 0)
        t = np.concatenate([u[1:], u[-1:]], 0)
    return cc * u + cw * w + ce * e + cs * s + cn * n + cb * b + ct * t


def _c2_like(shape, dtype, seed):
    """The C2 field shape: cos-product profile plus U[0, 1e-3) noise."""
    nz, ny, nx = shape
    cx = 1 - np.cos(2 * np.pi * np.arange(nx) / nx)
    cy = 1 - np.cos(2 * np.pi * np.arange(ny) / ny)
    cz = 1 - np.cos(2 * np.pi * np.arange(nz) / nz)
    f = 0.125 * cz[:, None, None] * cy[None, :, None] * cx[None, None, :]
    return (f + 1e-3 * np.random.default_rng(seed).random(shape)).astype(dtype)


def _run(f, steps, periodic=False, mode=ps.FP_FMA):
    ps.PSInit()
    ps.set_fp_mode(mode)
    try:
        return U.diffusion_gpu(f, steps, COEF, periodic=periodic, impl=ps.IMPL_TMA)
    finally:
        ps.set_fp_mode(ps.FP_EXACT)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("shape,field", [((40, 36, 130), "random"), ((33, 64, 64), "c2"),
                                         ((5, 7, 31), "random")])
def test_one_step_within_4_ulp(shape, field, periodic, dtype):
    f = (_c2_like(shape, dtype, 1) if field == "c2"
         else np.random.default_rng(1).random(shape).astype(dtype))
    exact = _exact_step(f, periodic)
    ref = oracle.diffusion7(f, 1, np.asarray(COEF, dtype), periodic=periodic)
    got = _run(f, 1, periodic)
    assert _ulp_err(got, exact) <= ULP_PER_STEP
    assert _ulp_err(ref, exact) <= ULP_PER_STEP  # the reference's result, same bar
    # and it really is the contracted form: some points differ from the exact mode
    if field == "random" and shape[0] > 8:
        assert not U.bits_equal(got, ref)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_each_step_within_4_ulp_of_the_exact_step(dtype):
    """Step by step over 12 steps: each FMA step, applied to the FMA run's own
    previous field, is within 4 ulp of the exact step from that field."""
    f = _c2_like((24, 40, 72), dtype, 2)
    for _ in range(12):
        exact = _exact_step(f, False)
        got = _run(f, 1)
        assert _ulp_err(got, exact) <= ULP_PER_STEP
        f = got


def test_many_steps_error_against_fp64_oracle():
    """200 steps of the C2 field at 64^3 against the FP64 oracle: the exact
    mode equals the reference bit for bit; the FMA run stays within the
    accumulated tolerance (4 ulp per step) and its error is of the same
    order as the exact run's (on this field it is about three times larger:
    the contracted sums round differently, not less often in effect)."""
    steps = 200
    f = _c2_like((64, 64, 64), np.float32, 3)
    ref64 = oracle.diffusion7_fp64(f, steps, COEF)
    exact = _run(f, steps, mode=ps.FP_EXACT)
    assert U.bits_equal(exact, oracle.diffusion7(f, steps, np.asarray(COEF, np.float32)))
    fast = _run(f, steps)
    e_exact = oracle.error_norms(exact, ref64)
    e_fast = oracle.error_norms(fast, ref64)
    assert e_fast["max_ulp_err"] <= ULP_PER_STEP * steps, e_fast
    assert e_fast["max_abs_err"] <= 10 * e_exact["max_abs_err"], (e_fast, e_exact)


def test_mode_switch_and_exact_default():
    ps.PSInit()
    assert ps.get_fp_mode() == ps.FP_EXACT
    with pytest.raises(ps.PhysisError):
        ps.set_fp_mode(7)
    f = np.random.default_rng(4).random((16, 24, 40)).astype(np.float32)
    want = oracle.diffusion7(f, 4, np.asarray(COEF, np.float32))
    _run(f, 4)  # FMA run, then back to exact: the exact run is bit-exact again
    assert U.bits_equal(U.diffusion_gpu(f, 4, COEF, impl=ps.IMPL_TMA), want)


# ---------------------------------------------------------------------------
# Generic tables compiled at run time (psb_generic_tma_compiled)
# ---------------------------------------------------------------------------
def _positive_table(rng, nterms, typ):
    """A read-times-constant table over one grid with positive coefficients
    (so partial sums grow and every rounding is at most half an ulp of the
    result), offsets within +-2, some terms unmultiplied."""
    terms = []
    for i in range(nterms):
        off = tuple(int(v) for v in rng.integers(-2, 3, size=3))
        if i % 5 == 3:
            terms.append(ps.get(0, off))
        else:
            terms.append((ps.const(float(np.float32(0.01 + 0.2 * rng.random()))), ps.get(0, off)))
    return ps.GenericStencil(3, [(typ, (0, 1, 2))] * 2, 1, typ, terms), terms


def _exact_generic(f, terms, lo, hi):
    """The table's value at every domain point in extended precision from the
    same inputs (coefficients rounded to the field's type)."""
    e = np.zeros(f.shape, dtype=np.longdouble)
    fx = f.astype(np.longdouble)
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    for t in terms:
        if t[0] == "g":
            c, g = np.longdouble(1), t
        else:
            c, g = np.longdouble(np.asarray(t[0][1], dtype=f.dtype)), t[1]
        dx, dy, dz = g[2]
        e[z0:z1, y0:y1, x0:x1] += c * fx[z0 + dz:z1 + dz, y0 + dy:y1 + dy, x0 + dx:x1 + dx]
    return e[z0:z1, y0:y1, x0:x1]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nterms", [5, 13, 27])
def test_generic_compiled_fma_within_the_rounding_bound(nterms, dtype):
    """FMA mode on a compiled packed table: one step from the same input lies
    within nterms/2 + 1 ulp of the extended-precision value (each of the
    nterms roundings is at most half an ulp of the growing positive sum),
    and the exact mode, switched back, equals the oracle port bit for bit."""
    ps.PSInit()
    rng = np.random.default_rng(40 + nterms)
    typ = ps.PS_FLOAT if dtype == np.float32 else ps.PS_DOUBLE
    st, terms = _positive_table(rng, nterms, typ)
    n = (52, 36, 30)
    f = (0.5 + 0.5 * rng.random(n[::-1])).astype(dtype)
    lo, hi = (2, 2, 2), (n[0] - 2, n[1] - 2, n[2] - 2)
    outs = {}
    try:
        for mode in (ps.FP_FMA, ps.FP_EXACT):
            ps.set_fp_mode(mode)
            g = [ps.grid_new(typ, n) for _ in range(2)]
            ps.PSGridCopyin(g[0], f)
            ps.PSGridCopyin(g[1], f)
            m = ps.PSStencilMap(st.kernel_id, ps.PSDomain3DNew(lo[0], hi[0], lo[1], hi[1], lo[2],
                                                               hi[2]), g[0], g[1])
            ps.PSStencilRun(m, 1)
            assert ps.generic_last_compiled()
            outs[mode] = ps.PSGridCopyout(g[1])
            for x in g:
                ps.PSGridFree(x)
    finally:
        ps.set_fp_mode(ps.FP_EXACT)
    exact = _exact_generic(f, terms, lo, hi)
    sl = (slice(lo[2], hi[2]), slice(lo[1], hi[1]), slice(lo[0], hi[0]))
    assert _ulp_err(outs[ps.FP_FMA][sl], exact) <= nterms / 2 + 1
    want = [f.copy(), f.copy()]
    oracle.generic_apply(st.struct, want, list(lo), list(hi))
    assert U.bits_equal(outs[ps.FP_EXACT], want[1])
    assert not U.bits_equal(outs[ps.FP_FMA], outs[ps.FP_EXACT])  # the modes differ
