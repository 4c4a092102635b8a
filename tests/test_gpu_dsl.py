"""Stencil functions compiled by the DSL front end, on the GPU.

Each system-test stencil, written as a DSL stencil function, is translated,
compiled for sm_100a and run through PSStencilMap / PSStencilRun; it must
print exactly what the reference's test_<name>.manual.ref.c prints."""
import numpy as np
import pytest

import physis_b200 as ps
from tests import gpu_util as U
from tests.golden import cases as C
from tests.golden import dsl_cases as D

CASES = dict(C.case_list(), **D.extra_cases())
DSL = D.dsl_cases()


@pytest.fixture(scope="module")
def kernels(tmp_path_factory):
    from physis_b200 import dsl
    ps.PSInit()
    seen, parts = set(), []
    for src, fn, _ in DSL.values():
        if fn not in seen:
            seen.add(fn)
            parts.append(src)
    return dsl.compile_stencils("\n".join(parts), str(tmp_path_factory.mktemp("dsl")))


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["staged", "own"])
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("name", sorted(DSL))
def test_compiled_stencil_matches_golden(name, layout, form, kernels):
    """Both forms of a compiled stencil print the reference's answer: the
    staged form (the function over the TMA plane ring) where the front end
    emitted one, and the stencil's own thread-per-point launch (forced with
    psb_set_impl(PSB_IMPL_GENERIC))."""
    src, fn, scalars = DSL[name]
    case = CASES[name]
    if form == "own":
        ps.set_impl(ps.IMPL_GENERIC)
    try:
        out = U.run_case_gpu(case, U.LAYOUTS[layout], kernel_id=kernels[fn].kernel_id,
                             params=scalars)
        ps.sync()
        staged = ps.compiled_last_staged()
    finally:
        ps.set_impl(ps.IMPL_AUTO)
    assert C.dump_text(out, case["fmt"]) == C.golden_text(name)
    want = _staged_form(kernels[fn].info, case, layout) if form == "staged" else 0
    assert staged == want, (name, layout, form)


def _staged_form(info, case, layout):
    """Which form the library runs for the last map of the case: 0 the
    function's own, 1 the staged form (every read range inside its grid over
    the domain), 2 the checked staged form (a read range may leave its grid,
    the domain lies inside every grid read). The staged forms need a
    function that has them, no red-black colour, the emitted grid not read,
    and pitched grids for periodic reads (their wrapped values come from the
    halo)."""
    if not info.staged:
        return 0
    slots, color = case["run"][-1]
    if color == 2:
        return 0
    if info.staged_periodic and layout != "pitched":
        return 0
    lo, hi = case["dom"]
    out = slots[info.emit_slot]
    inside = dom_inside = True
    for param, (rlo, rhi) in info.staged_reads.items():
        if slots[param] == out:
            return 0
        dims = case["grids"][slots[param]][1]
        if any(lo[k] + rlo[k] < 0 or hi[k] - 1 + rhi[k] > dims[k] - 1 for k in range(3)):
            inside = False
        if any(hi[k] > dims[k] for k in range(3)):
            dom_inside = False
    return 1 if inside else (2 if dom_inside else 0)


USER = D.user_cases()


def _run_user_case(case, layout_kernels):
    """A point-type case: records initialised as i + offset per component,
    the case's maps run, the dumped components printed like the reference's
    dump (one line per point, "%f" separated by spaces)."""
    n = C.N
    dims = (n, n, n)
    dt = case["dtype"]
    fields = []
    for name in dt.names:
        sub = dt.fields[name][0]
        count = int(np.prod(sub.shape)) if sub.shape else 1
        fields.append((ps.PS_FLOAT, count, dt.fields[name][1]))
    idx = np.arange(n ** 3, dtype=np.float64).reshape(n, n, n)
    recs = np.zeros((n, n, n), dt)
    for fname, flat, off in case["init"]:
        col = recs[fname].reshape(n, n, n, -1)
        col[..., flat] = 0 if off is None else (idx + off).astype(np.float32)
        recs[fname] = col.reshape(recs[fname].shape)
    grids = [ps.grid_new_user(dims, fields, dt.itemsize) for _ in range(case["grids"])]
    try:
        for g in grids:
            ps.user_copyin(g, recs)
        dom = ps.PSDomain3DNew(1, n - 1, 1, n - 1, 1, n - 1)
        maps = [ps.PSStencilMap(layout_kernels[fn].kernel_id, dom, *[grids[i] for i in slots])
                for fn, slots in case["steps"]]
        ps.PSStencilRun(*maps, case["iters"])
        out = np.zeros_like(recs)
        ps.user_copyout(grids[case["dump"]], out)
    finally:
        for g in grids:
            ps.PSGridFree(g)
    cols = [out[f].reshape(n ** 3, -1)[:, k] for f, k in case["comps"]]
    return "".join(" ".join("%f" % float(c[i]) for c in cols) + "\n" for i in range(n ** 3))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(USER))
def test_point_type_stencil_matches_golden(name, tmp_path):
    """The reference's user-defined point type tests, as DSL stencils over
    struct grids (member reads, whole-record emit, one-member emits)."""
    from physis_b200 import dsl
    case = USER[name]
    ks = dsl.compile_stencils(case["src"], str(tmp_path))
    assert _run_user_case(case, ks) == C.golden_text(name)


def _forms_run(form, fn):
    """fn() under the staged forms (the library's choice) or with the
    function's own launch forced; returns fn's result."""
    if form == "own":
        ps.set_impl(ps.IMPL_GENERIC)
    try:
        return fn()
    finally:
        ps.set_impl(ps.IMPL_AUTO)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["staged", "own"])
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
def test_read_outside_the_grid_is_reported_not_performed(tmp_path, form, layout):
    """x+1 at the last column and z-2 at the first two planes leave the grid:
    those reads return 0, nothing outside the grid is touched, and psb_sync
    reports PSB_ERR_BOUNDS, in the checked staged form as in the function's
    own form."""
    from physis_b200 import dsl
    k = dsl.compile_stencils("""
    void right(const int x, const int y, const int z, PSGrid3DFloat a, PSGrid3DFloat b) {
      PSGridEmit(b, PSGridGet(a, x + 1, y, z) + 2.0f * PSGridGet(a, x, y, z - 2) + 1.0f);
    }""", str(tmp_path))["right"]
    n = 16
    a = ps.grid_new(ps.PS_FLOAT, (n, n, n), U.LAYOUTS[layout])
    b = ps.grid_new(ps.PS_FLOAT, (n, n, n), U.LAYOUTS[layout])
    src = np.arange(n ** 3, dtype=np.float32).reshape(n, n, n)
    ps.PSGridCopyin(a, src)

    def run():
        ps.PSStencilRun(ps.PSStencilMap(k.kernel_id, ps.PSDomain3DNew(0, n, 0, n, 0, n), a, b), 1)
        with pytest.raises(ps.PhysisError) as e:
            ps.sync()
        return e.value.status, ps.compiled_last_staged()
    status, staged = _forms_run(form, run)
    assert status == ps.PSB_ERR_BOUNDS
    assert staged == (2 if form == "staged" else 0)
    ps.sync()  # the error word was cleared
    out = ps.PSGridCopyout(b)
    right = np.zeros_like(src)
    right[:, :, :-1] = src[:, :, 1:]
    down = np.zeros_like(src)
    down[2:] = src[:-2]
    expect = (right + np.float32(2) * down) + np.float32(1)
    assert np.array_equal(out, expect)
    for g in (a, b):
        ps.PSGridFree(g)


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["staged", "own"])
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("dims", [(40, 24, 20), (37, 29, 23), (5, 3, 4)])
def test_face_test_diffusion_matches_oracle(form, layout, dims):
    """The reference's 7-point diffusion kernel as written in the DSL (reads
    under face tests, examples/diffusion-benchmark/diffusion3d_physis.c:29-58)
    over the whole grid runs the checked staged form and equals the oracle's
    clamped diffusion bit for bit, like the function's own form; no read
    leaves the grid, so no error is reported."""
    from physis_b200 import dsl
    from physis_b200.workloads import DIFFUSION7_DSL
    from oracle import oracle as O
    k = dsl.compile_stencils(DIFFUSION7_DSL)["diffusion7"]
    coef = [0.1, 0.11, 0.12, 0.13, 0.14, 0.15, 0.25]  # ce cw cn cs ct cb cc
    field = np.random.default_rng(11).random(dims[::-1], dtype=np.float32)
    g = [ps.grid_new(ps.PS_FLOAT, dims, U.LAYOUTS[layout]) for _ in range(2)]
    ps.PSGridCopyin(g[0], field)
    d = ps.PSDomain3DNew(0, dims[0], 0, dims[1], 0, dims[2])

    def run():
        m1 = ps.PSStencilMap(k.kernel_id, d, g[0], g[1], *coef)
        m2 = ps.PSStencilMap(k.kernel_id, d, g[1], g[0], *coef)
        ps.PSStencilRun(m1, m2, 3)
        ps.sync()
        return ps.compiled_last_staged()
    staged = _forms_run(form, run)
    out = ps.PSGridCopyout(g[0])
    for x in g:
        ps.PSGridFree(x)
    # Dense rows and planes must be 16-byte multiples for TMA.
    tma = layout == "pitched" or (dims[0] % 4 == 0 and dims[0] * dims[1] % 4 == 0)
    assert staged == (2 if form == "staged" and tma else 0)
    assert U.bits_equal(out, O.diffusion7(field, 6, coef))


@pytest.mark.gpu
def test_in_place_update_needs_red_black(kernels):
    """A grid emitted and read off the point races without red-black order."""
    n = 8
    u = ps.grid_new(ps.PS_FLOAT, (n, n, n))
    dom = ps.PSDomain3DNew(1, n - 1, 1, n - 1, 1, n - 1)
    with pytest.raises(ps.PhysisError) as e:
        ps.PSStencilMap(kernels["rb7"].kernel_id, dom, u)
    assert e.value.status == ps.PSB_ERR_UNSUPPORTED
    ps.PSStencilMapRedBlack(kernels["rb7"].kernel_id, dom, u)
    ps.PSGridFree(u)


@pytest.mark.gpu
def test_compiled_matches_builtin_diffusion_in_graph_loop(kernels, tmp_path):
    """A long PSStencilRun (replayed as a CUDA graph) of a compiled 7-point
    diffusion equals the built-in kernel bit for bit."""
    from physis_b200 import dsl
    k = dsl.compile_stencils("""
    void diff(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat v,
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
    }""", str(tmp_path))["diff"]
    dims = (40, 24, 20)
    coef = [0.1, 0.11, 0.12, 0.13, 0.14, 0.15, 0.25]  # ce cw cn cs ct cb cc
    field = np.random.default_rng(3).random(dims[::-1], dtype=np.float32)
    ref = U.diffusion_gpu(field, 40, coef)
    g = [ps.grid_new(ps.PS_FLOAT, dims) for _ in range(2)]
    ps.PSGridCopyin(g[0], field)
    d = ps.PSDomain3DNew(0, dims[0], 0, dims[1], 0, dims[2])
    m1 = ps.PSStencilMap(k.kernel_id, d, g[0], g[1], *coef)
    m2 = ps.PSStencilMap(k.kernel_id, d, g[1], g[0], *coef)
    ps.PSStencilRun(m1, m2, 20)
    out = ps.PSGridCopyout(g[0])
    assert np.array_equal(out, ref)
    for x in g:
        ps.PSGridFree(x)


@pytest.mark.gpu
def test_point_type_transpose_with_loop_subscripts(tmp_path):
    """Members indexed by loop variables: b.p[j][i] = a(x, y, z).p[i][j]."""
    from physis_b200 import dsl
    k = dsl.compile_stencils("""
    struct M { float p[3][3]; };
    DeclareGrid3D(M, struct M);
    void transpose(const int x, const int y, const int z, PSGrid3DM a, PSGrid3DM b) {
      int i, j;
      for (i = 0; i < 3; i++)
        for (j = 0; j < 3; j++)
          PSGridEmitUtype(b.p[j][i], PSGridGet(a, x, y, z).p[i][j]);
    }""", str(tmp_path))["transpose"]
    dims = (12, 10, 8)
    dt = np.dtype([("p", np.float32, (3, 3))])
    recs = np.zeros(dims[::-1], dt)
    recs["p"] = np.random.default_rng(5).random(dims[::-1] + (3, 3), dtype=np.float32)
    a = ps.grid_new_user(dims, [(ps.PS_FLOAT, 9, 0)], dt.itemsize)
    b = ps.grid_new_user(dims, [(ps.PS_FLOAT, 9, 0)], dt.itemsize)
    try:
        ps.user_copyin(a, recs)
        dom = ps.PSDomain3DNew(0, dims[0], 0, dims[1], 0, dims[2])
        ps.PSStencilRun(ps.PSStencilMap(k.kernel_id, dom, a, b), 1)
        ps.sync()
        out = np.zeros_like(recs)
        ps.user_copyout(b, out)
    finally:
        ps.PSGridFree(a)
        ps.PSGridFree(b)
    assert np.array_equal(out["p"], np.swapaxes(recs["p"], -1, -2))


PERIODIC7_DSL = """
void wrapdiff(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat v,
              float ce, float cw, float cn, float cs, float ct, float cb, float cc) {
  float c = PSGridGet(u, x, y, z);
  float w = PSGridGetPeriodic(u, x - 1, y, z);
  float e = PSGridGetPeriodic(u, x + 1, y, z);
  float n = PSGridGetPeriodic(u, x, y - 1, z);
  float s = PSGridGetPeriodic(u, x, y + 1, z);
  float b = PSGridGetPeriodic(u, x, y, z - 1);
  float t = PSGridGetPeriodic(u, x, y, z + 1);
  PSGridEmit(v, cc * c + cw * w + ce * e + cs * s + cn * n + cb * b + ct * t);
}
"""

PERIODIC7_ONLY_DSL = PERIODIC7_DSL.replace("wrapdiff", "wrapdiff2").replace(
    "PSGridGet(u, x, y, z)", "PSGridGetPeriodic(u, x, y, z)")


@pytest.mark.gpu
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("dims", [(40, 24, 20), (37, 29, 23)])
def test_periodic_reads_staged_match_oracle(layout, dims, tmp_path):
    """A 7-point stencil whose neighbour reads wrap (PSGridGetPeriodic) runs
    staged on pitched grids -- the wrapped values come from the refreshed
    halo -- and equals the oracle's periodic diffusion bit for bit over a
    double-buffered run, whether its centre read is plain (wrapdiff) or
    periodic too (wrapdiff2); dense grids (no halo) keep the function's own
    form. The wrapped reads leave the grid's extent at its faces, so the
    checked staged form runs (it never checks a periodic read)."""
    from physis_b200 import dsl
    from oracle import oracle as O
    ks = dsl.compile_stencils(PERIODIC7_DSL + PERIODIC7_ONLY_DSL, str(tmp_path))
    assert ks["wrapdiff"].info.staged and ks["wrapdiff2"].info.staged
    coef = [0.1, 0.11, 0.12, 0.13, 0.14, 0.15, 0.25]  # ce cw cn cs ct cb cc
    field = np.random.default_rng(5).random(dims[::-1], dtype=np.float32)
    want = O.diffusion7(field, 6, coef, periodic=True)
    for name in ("wrapdiff", "wrapdiff2"):
        g = [ps.grid_new(ps.PS_FLOAT, dims, U.LAYOUTS[layout]) for _ in range(2)]
        try:
            ps.PSGridCopyin(g[0], field)
            d = ps.PSDomain3DNew(0, dims[0], 0, dims[1], 0, dims[2])
            m1 = ps.PSStencilMap(ks[name].kernel_id, d, g[0], g[1], *coef)
            m2 = ps.PSStencilMap(ks[name].kernel_id, d, g[1], g[0], *coef)
            ps.PSStencilRun(m1, m2, 3)
            ps.sync()
            staged = ps.compiled_last_staged()
            out = ps.PSGridCopyout(g[0])
        finally:
            for x in g:
                ps.PSGridFree(x)
        assert staged == (2 if layout == "pitched" else 0), (name, layout)
        assert U.bits_equal(out, want), (name, layout)
