"""Seeded workload inputs and single-grid runners over the public API.

Used by the benchmark, the smoke test and the parity tests alike: the
Himeno inputs of the C3-style configurations (the distributions of
examples/himeno/himenobmtxpa_physis.c:314-329) and two helpers that run a
double-buffered 7-point or Himeno solve through PSStencilMap/PSStencilRun
and return the result as a host array, the 27-point box table, and the
7-point stencil as DSL source for the front end. Everything here calls the
runtime library; nothing computes on the host.
"""
import numpy as np

import physis_b200 as ps


def himeno_inputs(shape, seed):
    """Seeded C3-style inputs: a0..a2, c0..c2 ~ U[0.9,1.1], a3 ~ U[0.95,1.05]/6,
    b0..b2 ~ U[-0.01,0.01], bnd 1 inside / 0 on faces, wrk1 = 0,
    p = (k/(nz-1))^2 (himenobmtxpa_physis.c:314-329)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    u = lambda lo, hi: (np.float32(lo) + np.float32(hi - lo) * rng.random(shape, dtype=np.float32))
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


def diffusion_gpu(field, steps, coef, periodic=False, impl=ps.IMPL_AUTO, layout=ps.LAYOUT_PITCHED,
                  dom=None, graph=True):
    """steps single updates (steps even: double-buffered PSStencilRun(m1, m2,
    steps/2)); returns the field."""
    t = ps.PS_FLOAT if field.dtype == np.float32 else ps.PS_DOUBLE
    nz, ny, nx = field.shape
    g1 = ps.grid_new(t, (nx, ny, nz), layout)
    g2 = ps.grid_new(t, (nx, ny, nz), layout)
    ps.PSGridCopyin(g1, field)
    if dom is None:
        d = ps.PSDomain3DNew(0, nx, 0, ny, 0, nz)
    else:
        d = ps.PSDomain3DNew(dom[0][0], dom[1][0], dom[0][1], dom[1][1], dom[0][2], dom[1][2])
    k = ps.DIFFUSION7_PERIODIC if periodic else ps.DIFFUSION7
    ps.set_impl(impl)
    ps.set_graph(graph)
    try:
        m1 = ps.PSStencilMap(k, d, g1, g2, *coef)
        m2 = ps.PSStencilMap(k, d, g2, g1, *coef)
        ps.PSStencilRun(m1, m2, steps // 2)
        if steps % 2:
            ps.PSStencilRun(m1, 1)
            out = ps.PSGridCopyout(g2)
        else:
            out = ps.PSGridCopyout(g1)
    finally:
        ps.set_impl(ps.IMPL_AUTO)
        ps.set_graph(True)
        ps.PSGridFree(g1)
        ps.PSGridFree(g2)
    return out


def himeno_gpu(p, coef, omega, sweeps, impl=ps.IMPL_AUTO, layout=ps.LAYOUT_PITCHED,
               residual=True):
    """sweeps (even) Himeno sweeps as PSStencilRun(m(p0->p1), m(p1->p0), sweeps/2).
    Returns (p, per-sweep gosa or None)."""
    nz, ny, nx = p.shape
    dims = (nx, ny, nz)
    gs = [ps.grid_new(ps.PS_FLOAT, dims, layout) for _ in range(14)]
    ps.PSGridCopyin(gs[0], p)
    ps.PSGridCopyin(gs[1], p)
    for i in range(12):
        ps.PSGridCopyin(gs[2 + i], coef[i])
    d = ps.PSDomain3DNew(1, nx - 1, 1, ny - 1, 1, nz - 1)
    ps.set_impl(impl)
    try:
        m1 = ps.PSStencilMap(ps.HIMENO19, d, *([gs[0], gs[1]] + gs[2:]), omega)
        m2 = ps.PSStencilMap(ps.HIMENO19, d, *([gs[1], gs[0]] + gs[2:]), omega)
        if residual:
            ps.himeno_residual_enable(m1, sweeps)
            ps.himeno_residual_enable(m2, sweeps)
        ps.PSStencilRun(m1, m2, sweeps // 2)
        out = ps.PSGridCopyout(gs[0])
        gosa = None
        if residual:
            h1 = ps.himeno_residual_history(m1, sweeps // 2)
            h2 = ps.himeno_residual_history(m2, sweeps // 2)
            gosa = [v for pair in zip(h1, h2) for v in pair]
    finally:
        ps.set_impl(ps.IMPL_AUTO)
        for g in gs:
            ps.PSGridFree(g)
    return out, gosa


def box27_offsets():
    """The 27 neighbour offsets in the order of the reference's
    tests/system_tests/test_cases/test_27-pt.c: z from -1 to 1, and in each
    plane the centre, then its ring (x+1, x-1, y+1 and its corners, y-1 and
    its corners)."""
    ring = [(0, 0), (1, 0), (-1, 0), (0, 1), (1, 1), (-1, 1), (0, -1), (1, -1), (-1, -1)]
    return [(dx, dy, dz) for dz in (-1, 0, 1) for dx, dy in ring]


def box27_terms(accum=ps.PS_FLOAT):
    """Terms of the 27-point box average: each neighbour times 1/27 (the
    float value for a float stencil, so that its double evaluation starts
    from the same coefficient)."""
    c = float(np.float32(1.0 / 27.0))
    return [(ps.const(c), ps.get(0, o)) for o in box27_offsets()]


def box27_struct(accum=ps.PS_FLOAT):
    """The 27-point box average as a psb_generic_stencil struct (unregistered:
    slot 0 read, slot 1 written)."""
    return ps.generic_struct(3, [(accum, (0, 1, 2))] * 2, 1, accum, box27_terms(accum))


def box27_stencil(accum=ps.PS_FLOAT):
    """The 27-point box average registered as a generic stencil."""
    return ps.GenericStencil(3, [(accum, (0, 1, 2))] * 2, 1, accum, box27_terms(accum))


# The 7-point diffusion of the C2 workload as a stencil function in the
# reference's DSL (the form of examples/diffusion-benchmark/diffusion3d_physis.c:
# clamped neighbours chosen at the faces, then the coefficient-weighted sum in
# the order cc, cw, ce, cs, cn, cb, ct), for the translator-free front end.
# Scalars follow the built-in kernel's order (ce, cw, cn, cs, ct, cb, cc), so
# the same PSStencilMap arguments drive either.
DIFFUSION7_DSL = """
void diffusion7(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat v,
                float ce, float cw, float cn, float cs, float ct, float cb, float cc) {
  const int nx = PSGridDim(u, 0), ny = PSGridDim(u, 1), nz = PSGridDim(u, 2);
  float c = PSGridGet(u, x, y, z);
  float w = x == 0 ? c : PSGridGet(u, x - 1, y, z);
  float e = x == nx - 1 ? c : PSGridGet(u, x + 1, y, z);
  float n = y == 0 ? c : PSGridGet(u, x, y - 1, z);
  float s = y == ny - 1 ? c : PSGridGet(u, x, y + 1, z);
  float b = z == 0 ? c : PSGridGet(u, x, y, z - 1);
  float t = z == nz - 1 ? c : PSGridGet(u, x, y, z + 1);
  PSGridEmit(v, cc * c + cw * w + ce * e + cs * s + cn * n + cb * b + ct * t);
}
"""


def _box27_dsl():
    def idx(v, d):
        return v if d == 0 else "%s %s %d" % (v, "+" if d > 0 else "-", abs(d))
    terms = " + ".join("c * PSGridGet(u, %s, %s, %s)" % (idx("x", dx), idx("y", dy), idx("z", dz))
                       for dx, dy, dz in box27_offsets())
    return ("void box27(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat v,\n"
            "           float c) {\n  PSGridEmit(v, %s);\n}\n" % terms)


# The 27-point box average as a DSL stencil function: the same terms, order
# and coefficient (passed as the scalar c = float(1/27)) as box27_terms, so
# over the interior [1, n-1)^3 it reads inside the grid everywhere and the
# front end's staged form runs it.
BOX27_DSL = _box27_dsl()
