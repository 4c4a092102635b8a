"""The generic stencil on the TMA z-streaming kernel (k_generic_tma), both as
the kernel that interprets the term table and as the kernel compiled at run
time for the table.

Every map the TMA path can take must give exactly what the thread-per-point
kernel and the oracle port give (the reference's term order and roundings):
the reference's system-test stencils (which run on the TMA path where they
are 3-D, single-type and not in place), random term tables with offsets up
to +-2 on every axis, constants and post factors, periodic and clamped reads
through the refreshed halo, several grids of different sizes, sub-domains,
float and double, and multi-step runs replayed from a CUDA graph.
"""
import ctypes

import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U
from tests.golden import cases as C

pytestmark = pytest.mark.gpu

CASES = C.case_list()
# Golden cases that fit the TMA path (3-D, one element type, reads within
# +-2, not in place, not red-black); periodic and clamped reads need the
# pitched layout's halo.
TMA_ANY = {"7-pt", "7-pt-multi-iterations", "7-pt-double-type", "27-pt", "asymmetric",
           "stencil-hole"}
TMA_PITCHED = TMA_ANY | {"7-pt-neumann-cond", "7-pt-periodic", "27-pt-periodic",
                         "asymmetric-periodic", "16", "3-pt-periodic"}


def last_impl():
    v = ctypes.c_int()
    ps.check(ps.lib.psb_generic_last_impl(ctypes.byref(v)), "psb_generic_last_impl")
    return v.value


@pytest.fixture(params=[True, False], ids=["compiled", "interpreted"])
def compile_mode(request):
    """Run the test with run-time compilation of packed tables on and off."""
    ps.PSInit()
    ps.set_generic_compile(request.param)
    yield request.param
    ps.set_generic_compile(True)


def _is_packed(st):
    """Every term one grid read times a constant (or a bare read), no post."""
    s = st.struct
    if s.has_post:
        return False
    return all((s.terms[i].a.grid >= 0) != (s.terms[i].b.grid >= 0) for i in range(s.nterms))


@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_cases_take_the_expected_kernel(name, layout, compile_mode):
    case = CASES[name]
    out = U.run_case_gpu(case, U.LAYOUTS[layout])
    assert C.dump_text(out, case["fmt"]) == C.golden_text(name)
    want = TMA_PITCHED if layout == "pitched" else TMA_ANY
    assert (last_impl() == ps.IMPL_TMA) == (name in want), (name, layout, last_impl())
    if last_impl() == ps.IMPL_TMA and not compile_mode:
        assert not ps.generic_last_compiled()


def _random_desc(rng, ngrids, typ, modes, nterms, post):
    """A random flat stencil over slots 0..ngrids-1 (read) writing slot
    ngrids; each read grid keeps one boundary form for all its reads."""
    axes = (0, 1, 2)
    terms = []
    for _ in range(nterms):
        g = int(rng.integers(0, ngrids))
        off = tuple(int(v) for v in rng.integers(-2, 3, size=3))
        a = ps.get(g, off, modes[g])
        r = rng.random()
        if r < 0.4:
            terms.append(a)
        elif r < 0.7:
            terms.append((ps.const(float(np.float32(rng.random() - 0.3))), a))
        else:
            g2 = int(rng.integers(0, ngrids))
            off2 = tuple(int(v) for v in rng.integers(-2, 3, size=3))
            terms.append((a, ps.get(g2, off2, modes[g2])))
    p = None
    if post == "const":
        p = ps.const(0.5)
    elif post == "grid":
        p = ps.get(0, (0, 0, 0), modes[0])
    return dict(ndims=3, grids=[(typ, axes)] * (ngrids + 1), out=ngrids, accum=typ, terms=terms,
                post=p)


def _run_both(d, arrays, dims_list, dom, layout, steps=1):
    """The map applied `steps` times on the TMA path and on the thread-per-
    point kernel; returns (tma result, plain result, impl of the TMA run)."""
    st = ps.GenericStencil(d["ndims"], d["grids"], d["out"], d["accum"], d["terms"], d.get("post"))
    outs, impl, compiled = [], None, None
    for mode in (ps.IMPL_AUTO, ps.IMPL_GENERIC):
        gs = [ps.grid_new(d["accum"], dims, layout) for dims in dims_list]
        try:
            for g, a in zip(gs, arrays):
                ps.PSGridCopyin(g, a)
            ps.set_impl(mode)
            dm = ps.PSDomain3DNew(dom[0][0], dom[1][0], dom[0][1], dom[1][1], dom[0][2], dom[1][2])
            m = ps.PSStencilMap(st.kernel_id, dm, *gs)
            ps.PSStencilRun(m, steps)
            if mode == ps.IMPL_AUTO:
                impl = last_impl()
                compiled = ps.generic_last_compiled()
            outs.append(ps.PSGridCopyout(gs[d["out"]]))
        finally:
            ps.set_impl(ps.IMPL_AUTO)
            for g in gs:
                ps.PSGridFree(g)
    return outs[0], outs[1], impl, st, compiled


SHAPES = [(37, 29, 41), (130, 9, 17), (5, 70, 6), (64, 64, 64)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("modes", ["none", "periodic", "clamp", "mixed"])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_tables_bit_exact(seed, modes, dtype, compile_mode):
    rng = np.random.default_rng(100 * seed + len(modes))
    typ = ps.PS_FLOAT if dtype == np.float32 else ps.PS_DOUBLE
    ngrids = 1 + seed % 3
    mlist = {"none": [ps.BOUNDARY_NONE] * 3, "periodic": [ps.BOUNDARY_PERIODIC] * 3,
             "clamp": [ps.BOUNDARY_CLAMP] * 3,
             "mixed": [ps.BOUNDARY_PERIODIC, ps.BOUNDARY_CLAMP, ps.BOUNDARY_NONE]}[modes]
    d = _random_desc(rng, ngrids, typ, mlist, int(rng.integers(3, 33)),
                     ("none", "const", "grid")[seed % 3])
    nx, ny, nz = SHAPES[seed + (1 if modes == "mixed" else 0)]
    dims_list = [(nx, ny, nz)] * (ngrids + 1)
    arrays = [(rng.random((nz, ny, nx)) - 0.2).astype(dtype) for _ in dims_list]
    # plain reads must stay inside the grid: the domain keeps 2 cells off the faces
    dom = ((2, 2, 2), (nx - 2, ny - 2, nz - 2)) if modes in ("none", "mixed") else \
        ((0, 0, 0), (nx, ny, nz))
    if min(h - l for l, h in zip(*dom)) <= 0:
        pytest.skip("grid too thin for plain reads")
    got, plain, impl, st, compiled = _run_both(d, arrays, dims_list, dom, ps.LAYOUT_PITCHED)
    assert impl == ps.IMPL_TMA
    assert compiled == compile_mode
    want = [a.copy() for a in arrays]
    oracle.generic_apply(st.struct, want, list(dom[0]), list(dom[1]))
    assert U.bits_equal(got, plain)
    assert U.bits_equal(got, want[ngrids])


def _random_packed_desc(rng, ngrids, typ, modes, nterms):
    """Every term one read (bare, or times a constant, which may be 1) of
    any of the grids at offsets within +-2: the form compiled at run time."""
    terms = []
    for _ in range(nterms):
        g = int(rng.integers(0, ngrids))
        off = tuple(int(v) for v in rng.integers(-2, 3, size=3))
        a = ps.get(g, off, modes[g])
        r = rng.random()
        if r < 0.3:
            terms.append(a)
        elif r < 0.4:
            terms.append((a, ps.const(1.0)))
        else:
            terms.append((ps.const(float(np.float32(rng.random() - 0.3))), a))
    return dict(ndims=3, grids=[(typ, (0, 1, 2))] * (ngrids + 1), out=ngrids, accum=typ,
                terms=terms)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("modes", ["none", "periodic", "clamp"])
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_random_packed_tables_compiled_bit_exact(seed, modes, dtype, compile_mode):
    """Read-times-constant tables of 1 to 32 terms over one to three grids:
    the compiled kernel (or, with compilation off, the interpreting one)
    equals the thread-per-point kernel and the oracle bit for bit."""
    rng = np.random.default_rng(700 + 10 * seed + len(modes))
    typ = ps.PS_FLOAT if dtype == np.float32 else ps.PS_DOUBLE
    ngrids = 1 + seed % 3
    mlist = {"none": [ps.BOUNDARY_NONE] * 3, "periodic": [ps.BOUNDARY_PERIODIC] * 3,
             "clamp": [ps.BOUNDARY_CLAMP] * 3}[modes]
    nterms = [1, 7, 19, 32][seed]
    d = _random_packed_desc(rng, ngrids, typ, mlist, nterms)
    nx, ny, nz = SHAPES[seed]
    dims_list = [(nx, ny, nz)] * (ngrids + 1)
    arrays = [(rng.random((nz, ny, nx)) - 0.2).astype(dtype) for _ in dims_list]
    dom = ((2, 2, 2), (nx - 2, ny - 2, nz - 2)) if modes == "none" else ((0, 0, 0), (nx, ny, nz))
    got, plain, impl, st, compiled = _run_both(d, arrays, dims_list, dom, ps.LAYOUT_PITCHED)
    assert impl == ps.IMPL_TMA and _is_packed(st)
    assert compiled == compile_mode
    want = [a.copy() for a in arrays]
    oracle.generic_apply(st.struct, want, list(dom[0]), list(dom[1]))
    assert U.bits_equal(got, plain)
    assert U.bits_equal(got, want[ngrids])


@pytest.mark.parametrize("layout,nx", [("pitched", 67), ("dense", 68), ("dense", 67)])
def test_27pt_sub_domain_and_dense_layout(layout, nx, compile_mode):
    """Sub-domains on both layouts. A dense grid takes the TMA path when its
    rows are a multiple of 16 bytes (68 floats); with 67-float rows it runs
    on the thread-per-point kernel, with the same result."""
    ny, nz = 33, 29
    f = np.random.default_rng(3).random((nz, ny, nx), dtype=np.float32)
    terms = [ps.get(0, o) for o in C._order27()]
    d = dict(ndims=3, grids=[(ps.PS_FLOAT, (0, 1, 2))] * 2, out=1, accum=ps.PS_FLOAT, terms=terms)
    for dom in [((1, 1, 1), (nx - 1, ny - 1, nz - 1)), ((5, 3, 7), (40, 30, 20)),
                ((1, 20, 1), (2, 21, 28))]:
        got, plain, impl, st, compiled = _run_both(d, [f, np.zeros_like(f)], [(nx, ny, nz)] * 2,
                                                   dom, U.LAYOUTS[layout])
        tma_ok = layout == "pitched" or nx * 4 % 16 == 0
        assert impl == (ps.IMPL_TMA if tma_ok else ps.IMPL_GENERIC)
        assert compiled == (tma_ok and compile_mode)
        want = [f.copy(), np.zeros_like(f)]
        oracle.generic_apply(st.struct, want, list(dom[0]), list(dom[1]))
        assert U.bits_equal(got, want[1]) and U.bits_equal(plain, want[1]), dom


def test_grids_of_different_sizes():
    """Two input grids larger than the output (as in a staggered map), with
    reads at positive offsets only into the larger grids."""
    ps.PSInit()
    n = (40, 24, 18)
    big = tuple(v + 2 for v in n)
    rng = np.random.default_rng(8)
    a, b = [rng.random(tuple(reversed(big)), dtype=np.float32) for _ in range(2)]
    terms = [(ps.get(0, (1, 1, 1)), ps.get(1, (2, 0, 1))), ps.get(1, (0, 2, 2)),
             (ps.const(0.25), ps.get(0, (2, 2, 0)))]
    d = dict(ndims=3, grids=[(ps.PS_FLOAT, (0, 1, 2))] * 3, out=2, accum=ps.PS_FLOAT, terms=terms)
    out0 = np.zeros(tuple(reversed(n)), np.float32)
    got, plain, impl, st, _ = _run_both(d, [a, b, out0], [big, big, n], ((0, 0, 0), n),
                                        ps.LAYOUT_PITCHED)
    assert impl == ps.IMPL_TMA
    want = [a.copy(), b.copy(), out0.copy()]
    oracle.generic_apply(st.struct, want, [0, 0, 0], list(n))
    assert U.bits_equal(got, want[2]) and U.bits_equal(plain, want[2])


@pytest.mark.parametrize("boundary", [ps.BOUNDARY_PERIODIC, ps.BOUNDARY_CLAMP])
def test_multi_step_runs_refresh_the_halo(boundary, compile_mode):
    """PSStencilRun(m(A->B), m(B->A), k): each map reads the grid the other
    just wrote, so its halo is refreshed before every step (also inside the
    replayed graph)."""
    nx, ny, nz = 48, 20, 26
    f = np.random.default_rng(11).random((nz, ny, nx), dtype=np.float32)
    offs = [(0, 0, 0), (2, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -2, 0), (0, 0, 1), (0, 0, -2),
            (1, 1, -1)]
    terms = [(ps.const(float(np.float32(0.1 + 0.01 * i))), ps.get(0, o, boundary))
             for i, o in enumerate(offs)]
    d = dict(ndims=3, grids=[(ps.PS_FLOAT, (0, 1, 2))] * 2, out=1, accum=ps.PS_FLOAT, terms=terms)
    st = ps.GenericStencil(3, d["grids"], 1, ps.PS_FLOAT, terms)
    g = [ps.grid_new(ps.PS_FLOAT, (nx, ny, nz)) for _ in range(2)]
    try:
        ps.PSGridCopyin(g[0], f)
        dom = ps.PSDomain3DNew(0, nx, 0, ny, 0, nz)
        m1 = ps.PSStencilMap(st.kernel_id, dom, g[0], g[1])
        m2 = ps.PSStencilMap(st.kernel_id, dom, g[1], g[0])
        ps.PSStencilRun(m1, m2, 7)
        assert last_impl() == ps.IMPL_TMA
        assert ps.generic_last_compiled() == compile_mode
        got = ps.PSGridCopyout(g[0])
    finally:
        for x in g:
            ps.PSGridFree(x)
    a, b = f.copy(), np.zeros_like(f)
    for _ in range(7):
        oracle.generic_apply(st.struct, [a, b], [0, 0, 0], [nx, ny, nz])
        oracle.generic_apply(st.struct, [b, a], [0, 0, 0], [nx, ny, nz])
    assert U.bits_equal(got, a)


def test_without_device_headers_the_interpreting_kernel_runs(tmp_path):
    """Run-time compilation needs the library's device headers; pointed at a
    directory without them it fails quietly and the interpreting kernel runs
    the same table with the same results (in a fresh process, so the
    function cache starts empty)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = r'''
import numpy as np
import physis_b200 as ps
from physis_b200.workloads import box27_stencil
from oracle import oracle
ps.PSInit()
st = box27_stencil(ps.PS_FLOAT)
n = 40
f = np.random.default_rng(2).random((n, n, n), dtype=np.float32)
g = [ps.grid_new(ps.PS_FLOAT, (n, n, n)) for _ in range(2)]
ps.PSGridCopyin(g[0], f)
ps.PSGridCopyin(g[1], f)
m = ps.PSStencilMap(st.kernel_id, ps.PSDomain3DNew(1, n - 1, 1, n - 1, 1, n - 1), g[0], g[1])
ps.PSStencilRun(m, 1)
got = ps.PSGridCopyout(g[1])
want = [f.copy(), f.copy()]
oracle.generic_apply(st.struct, want, [1, 1, 1], [n - 1] * 3)
print("compiled", ps.generic_last_compiled())
print("exact", np.array_equal(got.view(np.uint32), want[1].view(np.uint32)))
'''
    env = dict(os.environ, PHYSIS_B200_CSRC=str(tmp_path), PYTHONPATH=root)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         cwd=root, timeout=600)
    assert out.returncode == 0, out.stderr
    assert "compiled False" in out.stdout and "exact True" in out.stdout, out.stdout
