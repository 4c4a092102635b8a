"""The GPU runtime against the reference's known-answer outputs.

Each system-test stencil of the reference runs through the C ABI (generic
term-table kernel, both grid layouts) and must print exactly what the
reference's test_<name>.manual.ref.c prints.
"""
import pytest

from tests import gpu_util as U
from tests.golden import cases as C

CASES = C.case_list()


@pytest.mark.gpu
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_golden(name, layout):
    case = CASES[name]
    out = U.run_case_gpu(case, U.LAYOUTS[layout])
    assert C.dump_text(out, case["fmt"]) == C.golden_text(name)


@pytest.mark.gpu
@pytest.mark.parametrize("layout", sorted(U.LAYOUTS))
@pytest.mark.parametrize("impl", ["plain", "tma"])
def test_builtin_diffusion_matches_neumann_golden(impl, layout):
    """test_7-pt-neumann-cond through the built-in 7-point kernel."""
    import physis_b200 as ps
    case = CASES["7-pt-neumann-cond"]
    field = C.init_array("ramp", ps.PS_FLOAT, (C.N, C.N, C.N))
    coef = [float(c) for c in C.neumann_coefficients()]
    out = U.diffusion_gpu(field, 10, coef, impl={"plain": ps.IMPL_PLAIN, "tma": ps.IMPL_TMA}[impl],
                          layout=U.LAYOUTS[layout])
    assert C.dump_text(out, "%f") == C.golden_text("7-pt-neumann-cond")
