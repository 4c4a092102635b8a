"""Helpers shared by the GPU parity tests (run through the C ABI)."""
import numpy as np

import physis_b200 as ps
# Workload inputs and single-grid GPU runners live in the package (the
# benchmark and the smoke test use them too); re-exported for the tests.
from physis_b200.workloads import diffusion_gpu, himeno_gpu, himeno_inputs  # noqa: F401
from tests.golden import cases as C

LAYOUTS = {"pitched": ps.LAYOUT_PITCHED, "dense": ps.LAYOUT_DENSE}


def run_case_gpu(case, layout, kernel_id=None, params=()):
    """Execute one system-test case on the GPU with its generic descriptor
    (or the given kernel and scalars); returns the dumped array."""
    grids = []
    for kind, (t, dims) in zip(case["init"], case["grids"]):
        g = ps.grid_new(t, dims, layout)
        ps.PSGridCopyin(g, C.init_array(kind, t, dims))
        grids.append(g)
    if kernel_id is None:
        d = case["desc"]
        kernel_id = ps.GenericStencil(d["ndims"], d["grids"], d["out"], d["accum"], d["terms"],
                                      d.get("post")).kernel_id
    lo, hi = case["dom"]
    nd = len(lo)
    dom = [ps.PSDomain1DNew, ps.PSDomain2DNew, ps.PSDomain3DNew][nd - 1](
        *[v for pair in zip(lo, hi) for v in pair])
    maps = []
    for slots, color in case["run"]:
        args = [grids[s] for s in slots]
        if color == 2:
            maps.append(ps.PSStencilMapRedBlack(kernel_id, dom, *args, *params))
        else:
            maps.append(ps.PSStencilMap(kernel_id, dom, *args, *params))
    ps.PSStencilRun(*maps, case["iters"])
    out = ps.PSGridCopyout(grids[case["dump"]])
    for g in grids:
        ps.PSGridFree(g)
    return out


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(
        a.view(np.uint8), b.view(np.uint8))
