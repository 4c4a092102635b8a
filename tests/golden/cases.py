"""The reference's system-test stencils as generic-descriptor cases.

Each case restates one tests/system_tests/test_cases/test_<name>.c of the
reference: its grids, ramp inputs (indata[i] = i), domain, the terms of its
stencil function in source order, the PSStencilRun structure and the grid it
dumps. The expected output is the reference's hand-written known-answer
program test_<name>.manual.ref.c, whose stdout is committed (xz) next to this
file by make_golden.py. Both the oracle port (CPU) and the GPU runtime are
checked against those bytes.
"""
import lzma
import os

import numpy as np

from physis_b200 import (BOUNDARY_CLAMP as C, BOUNDARY_NONE as NB, BOUNDARY_PERIODIC as P,
                         PS_DOUBLE, PS_FLOAT, PS_INT, const, generic_struct, get)

HERE = os.path.dirname(os.path.abspath(__file__))
N = 32

XYZ = (0, 1, 2)


def _g(o, b=NB, slot=0):
    return get(slot, o, b)


ORDER7 = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, -1), (0, 0, 1)]
ORDER7_P = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


def _order27():
    out = []
    for dz in (-1, 0, 1):
        for (dx, dy) in [(0, 0), (1, 0), (-1, 0), (0, 1), (1, 1), (-1, 1), (0, -1), (1, -1),
                         (-1, -1)]:
            out.append((dx, dy, dz))
    return out


def _halo_dom(nd, h, n=N):
    return [h] * nd, [n - h] * nd


def neumann_coefficients():
    """ce..cc exactly as test_7-pt-neumann-cond.c computes them in C
    (float variables, double literals 0.1 and 1.0)."""
    f = np.float32
    nx = ny = nz = N
    l = f(1.0)
    kappa = f(0.1)
    dx, dy, dz = f(l / f(nx)), f(l / f(ny)), f(l / f(nz))
    dt = f(0.1 * np.float64(dx) * np.float64(dx) / np.float64(kappa))
    ce = cw = f(f(kappa * dt) / f(dx * dx))
    cn = cs = f(f(kappa * dt) / f(dy * dy))
    ct = cb = f(f(kappa * dt) / f(dz * dz))
    ssum = f(f(f(f(f(ce + cw) + cn) + cs) + ct) + cb)
    cc = f(1.0 - np.float64(ssum))
    return [ce, cw, cn, cs, ct, cb, cc]


def _neumann_terms():
    ce, cw, cn, cs, ct, cb, cc = neumann_coefficients()
    # cc*c + cw*w + ce*e + cs*s + cn*n + cb*b + ct*t with clamped neighbours
    pairs = [(cc, (0, 0, 0)), (cw, (-1, 0, 0)), (ce, (1, 0, 0)), (cs, (0, 1, 0)),
             (cn, (0, -1, 0)), (cb, (0, 0, -1)), (ct, (0, 0, 1))]
    return [(const(float(c)), _g(o, C)) for c, o in pairs]


def case_list():
    """name -> dict(grids, init, desc, dom, run, dump, fmt)."""
    cases = {}
    f3 = (PS_FLOAT, XYZ)

    def simple(name, terms, dom, typ=PS_FLOAT, fmt="%f"):
        cases[name] = dict(
            grids=[(typ, (N, N, N)), (typ, (N, N, N))], init=["ramp", "ramp"],
            desc=dict(ndims=3, grids=[(typ, XYZ), (typ, XYZ)], out=1, accum=typ, terms=terms),
            dom=dom, run=[([0, 1], -1)], iters=1, dump=1, fmt=fmt)

    simple("7-pt", [_g(o) for o in ORDER7], _halo_dom(3, 1))
    cases["7-pt-multi-iterations"] = dict(
        grids=[(PS_FLOAT, (N, N, N))] * 2, init=["ramp", "ramp"],
        desc=dict(ndims=3, grids=[f3, f3], out=1, accum=PS_FLOAT, terms=[_g(o) for o in ORDER7]),
        dom=_halo_dom(3, 1), run=[([0, 1], -1), ([1, 0], -1)], iters=5, dump=0, fmt="%f")
    cases["7-pt-neumann-cond"] = dict(
        grids=[(PS_FLOAT, (N, N, N))] * 2, init=["ramp", "zero"],
        desc=dict(ndims=3, grids=[f3, f3], out=1, accum=PS_FLOAT, terms=_neumann_terms()),
        dom=([0, 0, 0], [N, N, N]), run=[([0, 1], -1), ([1, 0], -1)], iters=5, dump=0, fmt="%f")
    simple("7-pt-periodic", [_g(o, P) for o in ORDER7_P], ([0, 0, 0], [N, N, N]))
    simple("7-pt-double-type", [_g(o) for o in ORDER7], _halo_dom(3, 1), typ=PS_DOUBLE)
    simple("7-pt-int-type", [_g(o) for o in ORDER7], _halo_dom(3, 1), typ=PS_INT, fmt="%d")
    cases["7-pt-type-mix"] = dict(
        grids=[(PS_FLOAT, (N, N, N)), (PS_DOUBLE, (N, N, N)), (PS_INT, (N, N, N))],
        init=["ramp", "zero", "mod10"],
        desc=dict(ndims=3, grids=[f3, (PS_DOUBLE, XYZ), (PS_INT, XYZ)], out=1, accum=PS_DOUBLE,
                  terms=[_g(o) for o in ORDER7], post=get(2, (0, 0, 0))),
        dom=_halo_dom(3, 1), run=[([0, 1, 2], -1)], iters=1, dump=1, fmt="%f")
    simple("27-pt", [_g(o) for o in _order27()], _halo_dom(3, 1))
    simple("27-pt-periodic", [_g(o, P) for o in _order27()], ([0, 0, 0], [N, N, N]))
    simple("asymmetric", [_g((0, 0, 0)), _g((1, 0, 0)), _g((-2, 0, 0))], _halo_dom(3, 2))
    simple("asymmetric-periodic", [_g((0, 0, 0)), _g((-1, 0, 0)), _g((2, 0, 0), P)],
           _halo_dom(3, 2))
    simple("stencil-hole", [_g((0, 0, 0)), _g((2, 0, 0)), _g((-2, 0, 0))], _halo_dom(3, 2))
    simple("16", [_g(o, C) for o in [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, 1, 0), (0, -1, 0),
                                     (0, 0, -1), (0, 0, 1)]], ([0, 0, 0], [N, N, N]))
    simple("3-pt-periodic", [_g((0, 0, 0), P), _g((0, 0, 1), P), _g((0, 0, -1), P)],
           ([0, 0, 0], [N, N, N]))
    cases["3-pt-1d"] = dict(
        grids=[(PS_FLOAT, (N,))] * 2, init=["ramp", "ramp"],
        desc=dict(ndims=1, grids=[(PS_FLOAT, (0,))] * 2, out=1, accum=PS_FLOAT,
                  terms=[_g((-1, 0, 0)), _g((0, 0, 0)), _g((1, 0, 0))]),
        dom=([1], [N - 1]), run=[([0, 1], -1)], iters=1, dump=1, fmt="%f")
    cases["9-pt-2d"] = dict(
        grids=[(PS_FLOAT, (N, N))] * 2, init=["ramp", "ramp"],
        desc=dict(ndims=2, grids=[(PS_FLOAT, (0, 1))] * 2, out=1, accum=PS_FLOAT,
                  terms=[_g((a, b, 0)) for a, b in [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1),
                                                    (-1, -1), (1, -1), (-1, 1), (1, 1)]]),
        dom=([1, 1], [N - 1, N - 1]), run=[([0, 1], -1)], iters=1, dump=1, fmt="%f")
    k1 = (PS_FLOAT, (0,))
    cases["mixed-dim"] = dict(
        grids=[(PS_FLOAT, (N, N, N))] * 2 + [(PS_FLOAT, (N,))], init=["ramp", "ramp", "alt12"],
        desc=dict(ndims=3, grids=[f3, f3, k1], out=1, accum=PS_FLOAT,
                  terms=[(_g((0, 0, 0)), get(2, (0, 0, 0))), (_g((-1, 0, 0)), get(2, (-1, 0, 0))),
                         (_g((1, 0, 0)), get(2, (1, 0, 0)))]),
        dom=([1, 0, 0], [N - 1, N, N]), run=[([0, 1, 2], -1)], iters=1, dump=1, fmt="%f")
    cases["mixed-dim2"] = dict(
        grids=[(PS_FLOAT, (N, N, N))] * 2 + [(PS_FLOAT, (N,))] * 3,
        init=["ramp", "ramp", "alt12", "alt12", "alt12"],
        desc=dict(ndims=3, grids=[f3, f3, (PS_FLOAT, (0,)), (PS_FLOAT, (1,)), (PS_FLOAT, (2,))],
                  out=1, accum=PS_FLOAT,
                  terms=[_g((0, 0, 0)),
                         (_g((-1, 0, 0)), get(2, (-1, 0, 0))), (_g((1, 0, 0)), get(2, (1, 0, 0))),
                         (_g((0, -1, 0)), get(3, (0, -1, 0))), (_g((0, 1, 0)), get(3, (0, 1, 0))),
                         (_g((0, 0, -1)), get(4, (0, 0, -1))), (_g((0, 0, 1)), get(4, (0, 0, 1)))]),
        dom=_halo_dom(3, 1), run=[([0, 1, 2, 3, 4], -1)], iters=1, dump=1, fmt="%f")
    cases["mixed-dim3"] = dict(
        grids=[(PS_FLOAT, (N, N + 2, N))] * 2 + [(PS_FLOAT, (N,)), (PS_FLOAT, (N + 2, N))],
        init=["ramp", "ramp", "alt12", "alt12"],
        desc=dict(ndims=3, grids=[f3, f3, (PS_FLOAT, (0,)), (PS_FLOAT, (1, 2))], out=1,
                  accum=PS_FLOAT,
                  terms=[_g((0, 0, 0)),
                         (_g((-1, 0, 0)), get(2, (-1, 0, 0))), (_g((1, 0, 0)), get(2, (1, 0, 0))),
                         (_g((0, -1, 0)), get(3, (0, -1, 0))), (_g((0, 1, 0)), get(3, (0, 1, 0))),
                         (_g((0, 0, -1)), get(3, (0, 0, -1))), (_g((0, 0, 1)), get(3, (0, 0, 1)))]),
        dom=([1, 1, 1], [N - 1, N + 1, N - 1]), run=[([0, 1, 2, 3], -1)], iters=1, dump=1,
        fmt="%f")
    cases["redblack"] = dict(
        grids=[(PS_FLOAT, (N, N, N))], init=["ramp"],
        desc=dict(ndims=3, grids=[f3], out=0, accum=PS_FLOAT, terms=[_g(o) for o in ORDER7]),
        dom=_halo_dom(3, 1), run=[([0], 2)], iters=1, dump=0, fmt="%f")
    cases["redblack-periodic"] = dict(
        grids=[(PS_FLOAT, (N, N, N))], init=["ramp"],
        desc=dict(ndims=3, grids=[f3], out=0, accum=PS_FLOAT,
                  terms=[_g(o, P) for o in ORDER7]),
        dom=([0, 0, 0], [N, N, N]), run=[([0], 2)], iters=1, dump=0, fmt="%f")
    return cases


def init_array(kind, typ, dims):
    shape = tuple(reversed(dims))
    n = int(np.prod(dims))
    dt = {PS_FLOAT: np.float32, PS_DOUBLE: np.float64, PS_INT: np.int32}[typ]
    if kind == "ramp":
        a = np.arange(n, dtype=np.float64)
    elif kind == "zero":
        a = np.zeros(n)
    elif kind == "mod10":
        a = np.arange(n) % 10
    elif kind == "alt12":
        a = 1 + (np.arange(n) % 2)
    else:
        raise ValueError(kind)
    return a.astype(dt).reshape(shape)


def descriptor(case):
    d = case["desc"]
    return generic_struct(d["ndims"], d["grids"], d["out"], d["accum"], d["terms"],
                          d.get("post"))


def dump_text(arr, fmt):
    flat = np.asarray(arr).ravel()
    if fmt == "%d":
        return "".join("%d\n" % int(v) for v in flat)
    return "".join("%f\n" % float(v) for v in flat)


def golden_text(name):
    with lzma.open(os.path.join(HERE, name + ".txt.xz"), "rt") as f:
        return f.read()


def run_oracle(case):
    """Execute a case with the oracle port; returns the dumped array."""
    from oracle import oracle
    arrays = [init_array(k, t, d) for k, (t, d) in zip(case["init"], case["grids"])]
    desc = descriptor(case)
    lo, hi = case["dom"]
    for _ in range(case["iters"]):
        for slots, color in case["run"]:
            view = [arrays[s] for s in slots]
            if color == 2:
                oracle.generic_apply(desc, view, lo, hi, 0)
                oracle.generic_apply(desc, view, lo, hi, 1)
            else:
                oracle.generic_apply(desc, view, lo, hi, color)
    return arrays[case["dump"]]
