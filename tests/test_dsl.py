"""The DSL front end on the CPU: translation, DSL rule checks and an sm_100a
cross-compile of the generated kernels (nothing here needs a GPU)."""
import ctypes
import glob
import os

import pytest

import physis_b200 as ps
from physis_b200 import dsl
from tests.golden import dsl_cases as D

# The reference's system tests, where the reference tree is present (this
# CPU test is skipped elsewhere).
REF_TESTS = os.path.join(os.environ.get("PHYSIS_REFERENCE", "/root/reference"),
                         "tests", "system_tests", "test_cases")


def _all_case_source():
    seen, parts = set(), []
    for src, fn, _ in D.dsl_cases().values():
        if fn not in seen:
            seen.add(fn)
            parts.append(src)
    return "\n".join(parts)


def test_translation_metadata():
    _, infos = dsl.translate(_all_case_source())
    k = infos["sum7"]
    assert k.ndims == 3 and k.grid_types == [ps.PS_FLOAT, ps.PS_FLOAT]
    assert k.emits == [0, 1] and k.reads_offset == [1, 0]
    n = infos["neumann7"]
    assert [t for _, t in n.scalars] == [ps.PS_FLOAT] * 7
    m = infos["weighted_planes"]
    assert [nd for _, _, nd in m.grids] == [3, 3, 1, 2]
    assert m.axes[2] == [0] and m.axes[3] == [1, 2]
    assert infos["line3"].ndims == 1 and infos["plane9"].ndims == 2
    rb = infos["rb7"]
    assert rb.emits == [1] and rb.reads_offset == [1]
    mix = infos["mixed_types"]
    assert mix.grid_types == [ps.PS_FLOAT, ps.PS_DOUBLE, ps.PS_INT] and mix.emits == [0, 1, 0]


def test_generated_code_keeps_c_semantics():
    src = """
    #define SCALE 0.5
    void f(const int x, const int y, const int z, PSGrid3DFloat a, PSGrid3DFloat b, float t) {
      float v = PSGridGet(a, x, y, z) / 7.0 * t;
      PSGridEmit(b, sqrt(v) * SCALE + fabsf(v));
    }
    """
    cu, infos = dsl.translate(src)
    assert "sqrt((double) v)" in cu          # C promotes the float argument
    assert "fabsf(v)" in cu                  # the float function stays as written
    assert "0.5" in cu and "SCALE" not in cu  # the source's own macros are expanded
    assert "__psb_emit(b, x, y, z" in cu


@pytest.mark.parametrize("src, msg", [
    ("void f(PSGrid3DFloat a, const int x) { }", "no stencil function"),
    ("void f(const int x, PSGrid1DFloat a, float *p) { PSGridEmit(a, 0); }", "parameters must"),
    ("void f(const int x, PSGrid1DFloat a, PSGrid1DFloat b) { float v = PSGridGet(3, x); }",
     "grid parameter"),
    ("void f(const int x, const int y, PSGrid2DFloat a, PSGrid1DFloat b) { PSGridEmit(b, 1); }",
     "PSGridEmit into a 1-D grid"),
    ("void f(const int x, PSGrid1DFloat a, PSGrid1DFloat b) { PSGridEmit(b, PSGridGet(a, x, x)); }",
     "takes 1 indices"),
    ("float h(PSGrid1DFloat a, int i) { return 0; }\n"
     "void f(const int x, PSGrid1DFloat a, PSGrid1DFloat b) { PSGridEmit(b, h(a, x)); }",
     "begins with its `const int` index"),
    ("struct P { float u; };\nDeclareGrid1D(P, struct P);\n"
     "void f(const int x, PSGrid1DP a) { PSGridEmitUtype(a.v, 1.0f); }", "has no member v"),
    ("struct P { float u[2]; };\nDeclareGrid1D(P, struct P);\n"
     "void f(const int x, PSGrid1DP a) { PSGridEmitUtype(a.u, 1.0f); }", "give all 1 subscripts"),
    ("struct P { float u; };\nDeclareGrid1D(P, struct P);\n"
     "void f(const int x, PSGrid1DP a) { float v = a.u; }", "only written by PSGridEmitUtype"),
    ("void f(const int x, PSGrid1DFloat a) { void *p = &a; }", "address of a grid"),
    ("void f(const int x, PSGrid1DFloat a) { PSGridCopyin(a, 0); }", "not available"),
    ("int f(const int x, PSGrid1DFloat a) { return 0; }", "return void"),
    ("void f(const int x, PSGrid1DFloat a) { float v = ; }", "cannot parse"),
])
def test_dsl_rule_violations_are_reported(src, msg):
    with pytest.raises(dsl.DSLError, match=msg):
        dsl.translate(src)


def test_generated_library_builds_for_sm100a(tmp_path):
    """nvcc compiles every case's kernel; the library exports the launch and
    describe functions of each stencil, and the descriptions match."""
    cu, infos = dsl.translate(_all_case_source())
    so = dsl.build_library(cu, str(tmp_path))
    lib = ctypes.CDLL(so)
    for name, info in infos.items():
        assert hasattr(lib, "psb_dsl_launch_" + name)
        d = ps.CompiledStencilStruct()
        getattr(lib, "psb_dsl_describe_" + name)(ctypes.byref(d))
        assert d.ndims == info.ndims and d.ngrids == len(info.grids)
        assert list(d.grid_type)[:d.ngrids] == info.grid_types
        assert d.nviews == len(info.view_type)
        assert list(d.view_type)[:d.nviews] == info.view_type
        assert list(d.view_emits)[:d.nviews] == info.view_emits
        assert list(d.view_reads_offset)[:d.nviews] == info.view_reads_offset
        assert d.nparams == len(info.scalars) and d.launch
        # The staged forms: both entry points or neither, the read ranges and
        # the periodic flags of the grids the form reads.
        assert bool(d.staged) == info.staged and bool(d.staged_checked) == info.staged
        for slot in range(d.ngrids):
            r = info.staged_reads.get(slot) if info.staged else None
            lo, hi = list(d.read_lo[slot]), list(d.read_hi[slot])
            if r is None:
                assert lo[0] > hi[0] and not d.read_periodic[slot], (name, slot)
            else:
                assert [lo, hi] == r, (name, slot)
                assert d.read_periodic[slot] == (slot in info.staged_periodic), (name, slot)


def test_staged_form_eligibility():
    """Which functions get staged forms: constant offsets within +-2, one
    top-level emit into a grid not read; reads under face tests (checked at
    run time) and periodic reads (from the halo), alone or mixed, qualify;
    offsets beyond the halo, reads at run-time offsets and a read of the
    emitted grid do not."""
    src = """
    void faces(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat v) {
      float c = PSGridGet(u, x, y, z);
      float w = x == 0 ? c : PSGridGet(u, x - 1, y, z);
      PSGridEmit(v, c + w);
    }
    void wrap(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat v) {
      PSGridEmit(v, PSGridGetPeriodic(u, x - 2, y, z) + PSGridGet(u, x, y, z + 1));
    }
    void far(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat v) {
      PSGridEmit(v, PSGridGet(u, x + 3, y, z));
    }
    void moving(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat v,
                int k) {
      PSGridEmit(v, PSGridGet(u, x + k, y, z));
    }
    void inplace(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat v) {
      PSGridEmit(v, PSGridGet(v, x, y, z) + PSGridGet(u, x, y, z));
    }
    """
    _, infos = dsl.translate(src)
    assert infos["faces"].staged and not infos["faces"].staged_periodic
    assert infos["faces"].staged_reads == {0: [[-1, 0, 0], [0, 0, 0]]}
    assert infos["wrap"].staged and infos["wrap"].staged_periodic == {0}
    assert infos["wrap"].staged_reads == {0: [[-2, 0, 0], [0, 0, 1]]}
    assert not infos["far"].staged
    assert not infos["moving"].staged
    assert not infos["inplace"].staged


@pytest.mark.skipif(not os.path.isdir(REF_TESTS), reason="reference sources not present")
def test_reference_system_tests_translate():
    """Every stencil function of the reference's system tests translates,
    the user-defined point types included."""
    done = 0
    for f in sorted(glob.glob(os.path.join(REF_TESTS, "test_*.c"))):
        if ".manual." in f:
            continue
        text = open(f).read()
        if "PSGridEmit" not in text:
            continue
        _, infos = dsl.translate(text)
        assert infos, f
        done += 1
    assert done >= 33


@pytest.mark.skipif(not os.path.isdir(REF_TESTS), reason="reference sources not present")
def test_reference_system_tests_compile_for_sm100a(tmp_path):
    """The translation of every reference system test with a stencil builds
    with nvcc for sm_100a (host cross-compile, no GPU)."""
    import concurrent.futures
    files = [f for f in sorted(glob.glob(os.path.join(REF_TESTS, "test_*.c")))
             if ".manual." not in f and "PSGridEmit" in open(f).read()]

    def build(f):
        cu, _ = dsl.translate(open(f).read())
        return dsl.build_library(cu, str(tmp_path))

    with concurrent.futures.ThreadPoolExecutor(max_workers=8) as ex:
        libs = list(ex.map(build, files))
    assert len(libs) == len(files) >= 33 and all(os.path.exists(p) for p in libs)


def test_point_type_views():
    """A grid of a point type is one view per scalar component (fields in
    order, arrays row-major); reads and emits are tracked per component."""
    _, infos = dsl.translate(D.user_cases()["user-defined-type-multi-dim-member"]["src"])
    k = infos["corners"]
    assert k.grid_types == [ps.PS_USER] and k.view_type == [ps.PS_FLOAT] * 6
    assert k.view_emits == [0, 0, 1, 0, 0, 0]           # e[1][0]
    assert k.view_reads_offset == [1, 0, 0, 0, 0, 1]    # e[0][0] and e[2][1]
    _, infos = dsl.translate(D.user_cases()["user-defined-type1"]["src"])
    k = infos["smooth3"]
    assert k.view_emits == [0, 0, 0, 1, 1, 1] and k.view_reads_offset == [1, 1, 1, 0, 0, 0]


def test_run_time_member_subscripts_are_checked():
    """A member subscript computed at run time (a loop over a matrix member)
    goes through the checked helpers: outside the member it reads 0 or
    stores nothing and reports PSB_ERR_BOUNDS instead of indexing past the
    member's component list."""
    src = """
    struct M { float p[3][3]; };
    DeclareGrid3D(M, struct M);
    void transpose(const int x, const int y, const int z, PSGrid3DM a, PSGrid3DM b) {
      int i, j;
      for (i = 0; i < 3; i++)
        for (j = 0; j < 3; j++)
          PSGridEmitUtype(b.p[j][i], PSGridGet(a, x, y, z).p[i][j]);
    }
    """
    cu, infos = dsl.translate(src)
    assert "__psb_emit_c(b__p, 9, (j * 3) + i" in cu and "__psb_get_c(a__p, 9, (i * 3) + j" in cu
    k = infos["transpose"]
    assert k.view_emits == [0] * 9 + [1] * 9 and k.view_reads_offset == [0] * 18


def test_command_line_translation(tmp_path):
    """`python -m physis_b200.dsl src -o out.cu` writes the generated CUDA
    (translation only, no nvcc) and lists the stencil functions found."""
    import subprocess
    import sys
    src = tmp_path / "k.c"
    src.write_text(D.dsl_cases()["7-pt"][0])
    out = tmp_path / "k.cu"
    r = subprocess.run([sys.executable, "-m", "physis_b200.dsl", str(src), "-o", str(out)],
                       capture_output=True, text=True,
                       cwd=os.path.abspath(os.path.join(os.path.dirname(__file__), "..")))
    assert r.returncode == 0, r.stderr
    assert "sum7: 3-D" in r.stdout
    text = out.read_text()
    assert "__global__" in text and "psb_dsl_describe_sum7" in text
