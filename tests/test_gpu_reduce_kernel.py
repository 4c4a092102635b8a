"""Kernel-function reduction (PSReduce(&v, op, kernel, dom, ...), the form the
reference documents but does not implement): the values a generic stencil
would emit, reduced without being stored, against the oracle that applies
the stencil into an array and reduces it on the host."""
import math

import numpy as np
import pytest

import physis_b200 as ps
from oracle import oracle
from tests import gpu_util as U
from tests.golden import cases as C


def _factors(d):
    for t in d["terms"]:
        for f in ([t] if isinstance(t[0], str) else list(t)):
            yield f
    if d.get("post") is not None:
        yield d["post"]


def _eligible():
    """Golden cases whose first map emits a grid of the domain's dimension
    and does not read it at an offset (so the emitted values do not depend
    on the order in which points are written)."""
    out = []
    for name, case in sorted(C.case_list().items()):
        d = case["desc"]
        slots, color = case["run"][0]
        reads_out = any(f[0] == "g" and f[1] == d["out"] and any(f[2]) for f in _factors(d))
        full_dim = len(d["grids"][d["out"]][1]) == d["ndims"]
        if color == -1 and not reads_out and full_dim:
            out.append(dict(case, name=name))
    return out


CASES = _eligible()


def _expected(case):
    arrays = [C.init_array(k, t, dims) for k, (t, dims) in zip(case["init"], case["grids"])]
    desc = C.descriptor(case)
    lo, hi = case["dom"]
    slots, _ = case["run"][0]
    view = [arrays[s] for s in slots]
    oracle.generic_apply(desc, view, lo, hi, -1)
    emitted = view[case["desc"]["out"]]
    sel = tuple(slice(lo[k], hi[k]) for k in reversed(range(len(lo))))
    return np.ascontiguousarray(emitted[sel]).ravel()


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_kernel_reduction_matches_oracle(case):
    vals = _expected(case).astype(np.float64)
    grids = []
    for kind, (t, dims) in zip(case["init"], case["grids"]):
        g = ps.grid_new(t, dims)
        ps.PSGridCopyin(g, C.init_array(kind, t, dims))
        grids.append(g)
    try:
        d = case["desc"]
        st = ps.GenericStencil(d["ndims"], d["grids"], d["out"], d["accum"], d["terms"], d.get("post"))
        lo, hi = case["dom"]
        dom = [ps.PSDomain1DNew, ps.PSDomain2DNew, ps.PSDomain3DNew][len(lo) - 1](
            *[v for pair in zip(lo, hi) for v in pair])
        slots, _ = case["run"][0]
        args = [grids[s] for s in slots]
        assert ps.PSReduceMap(ps.PS_MAX, st.kernel_id, dom, *args) == vals.max()
        assert ps.PSReduceMap(ps.PS_MIN, st.kernel_id, dom, *args) == vals.min()
        got = ps.PSReduceMap(ps.PS_SUM, st.kernel_id, dom, *args)
        want = math.fsum(vals)
        assert abs(got - want) <= 1e-13 * float(np.abs(vals).sum()) + 1e-300
        # The grids are unchanged: nothing is stored.
        for kind, (t, dims), g in zip(case["init"], case["grids"], grids):
            assert U.bits_equal(ps.PSGridCopyout(g), C.init_array(kind, t, dims))
    finally:
        for g in grids:
            ps.PSGridFree(g)


def test_cases_are_selected():
    assert len(CASES) >= 5
