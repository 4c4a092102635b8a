"""Python access to the oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker: nothing in the physis_b200 product
path calls it.

Two CPU implementations are reachable from here:
  * the port -- oracle/port.c, a plain-C restatement of the reference CPU
    target's arithmetic (build/liboracle_port.so);
  * the reference itself -- libphysis_rt_ref compiled from the reference's
    runtime sources plus translator-shaped programs (oracle/ref_paths.c),
    in _ref/libphysis_ref_paths.so. It exists only where the reference
    sources were available when the oracle was built.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "build", "liboracle_port.so")
REF_LIB = os.path.join(HERE, "_ref", "libphysis_ref_paths.so")
REF_SRC = os.environ.get("PHYSIS_REFERENCE", "/root/reference")

PS_MAX, PS_MIN, PS_SUM, PS_PROD = 0, 1, 2, 3
PS_INT, PS_LONG, PS_FLOAT, PS_DOUBLE = 0, 1, 2, 3

_port = None
_ref = None


def build(with_ref=None):
    """Compile the port (always) and the reference runtime (when its sources
    are present). Returns (port_ok, ref_ok)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    if with_ref is None:
        with_ref = os.path.isdir(os.path.join(REF_SRC, "runtime"))
    ref_ok = os.path.exists(REF_LIB)
    if with_ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + REF_SRC], check=True)
        ref_ok = True
    return True, ref_ok


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            build(with_ref=False)
        lib = ctypes.CDLL(PORT_LIB)
        P = ctypes.c_void_p
        I = ctypes.c_int
        for name in ("orc_diffusion7_f32", "orc_diffusion7_f64"):
            f = getattr(lib, name)
            f.restype = None
            f.argtypes = [I, I, I, P, P, I, P, I, P, P]
        lib.orc_himeno_f32.restype = None
        lib.orc_himeno_f32.argtypes = [I, I, I, P, P, P, ctypes.c_float, I, P]
        lib.orc_himeno_f64.restype = None
        lib.orc_himeno_f64.argtypes = [I, I, I, P, P, P, ctypes.c_double, I, P]
        lib.orc_generic_apply.restype = None
        lib.orc_generic_apply.argtypes = [P, P, P, P, P, I]
        lib.orc_fold_f32.restype = None
        lib.orc_fold_f32.argtypes = [I, P, ctypes.c_int64, P]
        lib.orc_fold_f64.restype = None
        lib.orc_fold_f64.argtypes = [I, P, ctypes.c_int64, P]
        lib.orc_sum_f64.restype = None
        lib.orc_sum_f64.argtypes = [P, I, ctypes.c_int64, P, P]
        _port = lib
    return _port


def ref_available():
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        # DEEPBIND: the reference runtime exports the same C names as the B200
        # runtime (PSInit, __PSGridNew, ...); its programs must bind to it.
        lib = ctypes.CDLL(REF_LIB, mode=os.RTLD_LOCAL | os.RTLD_DEEPBIND)
        P = ctypes.c_void_p
        I = ctypes.c_int
        lib.refp_init.restype = None
        lib.refp_init.argtypes = []
        for name in ("refp_diffusion7_f32", "refp_diffusion7_f64"):
            f = getattr(lib, name)
            f.restype = ctypes.c_double
            f.argtypes = [I, I, I, P, I, P, I]
        lib.refp_himeno_f32.restype = ctypes.c_double
        lib.refp_himeno_f32.argtypes = [I, I, I, P, P, ctypes.c_float, I]
        lib.refp_box27_f32.restype = ctypes.c_double
        lib.refp_box27_f32.argtypes = [I, I, I, P, I, ctypes.c_float]
        lib.refp_reduce_f32.restype = None
        lib.refp_reduce_f32.argtypes = [I, P, ctypes.c_int64, P]
        lib.refp_reduce_f64.restype = None
        lib.refp_reduce_f64.argtypes = [I, P, ctypes.c_int64, P]
        lib.refp_init()
        _ref = lib
    return _ref


def _ptr(a):
    return a.ctypes.data if a is not None else None


# ---------------------------------------------------------------------------
# Port entry points
# ---------------------------------------------------------------------------
def diffusion7(field, steps, coef, periodic=False, lo=None, hi=None):
    """steps single 7-point updates of field (shape (nz, ny, nx)); coef is
    (ce, cw, cn, cs, ct, cb, cc). Returns the new field."""
    dt = field.dtype
    a = np.array(field, dtype=dt, copy=True, order="C")
    b = np.zeros_like(a)
    c = np.asarray(coef, dtype=dt)
    nz, ny, nx = a.shape
    f = port().orc_diffusion7_f32 if dt == np.float32 else port().orc_diffusion7_f64
    lo_a = np.asarray(lo, dtype=np.int32) if lo is not None else None
    hi_a = np.asarray(hi, dtype=np.int32) if hi is not None else None
    f(nx, ny, nz, _ptr(a), _ptr(b), steps, _ptr(c), 1 if periodic else 0, _ptr(lo_a), _ptr(hi_a))
    return a


def himeno(p, coef, omega, sweeps):
    """sweeps Himeno updates. coef: 12 arrays a0 a1 a2 a3 b0 b1 b2 c0 c1 c2 bnd
    wrk1. p1 starts as a copy of p. Returns (final p after the sweeps, gosa
    per sweep)."""
    a = np.array(p, dtype=np.float32, copy=True)
    b = a.copy()
    cs = [np.ascontiguousarray(c, dtype=np.float32) for c in coef]
    arr = (ctypes.c_void_p * 12)(*[c.ctypes.data for c in cs])
    gosa = np.zeros(max(1, sweeps), dtype=np.float64)
    nz, ny, nx = a.shape
    port().orc_himeno_f32(nx, ny, nz, _ptr(a), _ptr(b), ctypes.cast(arr, ctypes.c_void_p),
                          ctypes.c_float(omega), sweeps, _ptr(gosa))
    return (a if sweeps % 2 == 0 else b), gosa[:sweeps]


# ---------------------------------------------------------------------------
# FP64 oracle: the same algorithms, term order and inputs, in double
# ---------------------------------------------------------------------------
def diffusion7_fp64(field, steps, coef, periodic=False):
    """The 7-point run of diffusion7() in double from the same inputs: the
    field and the coefficients are the fp32 (or fp64) values, widened."""
    c = np.asarray(coef, dtype=field.dtype).astype(np.float64)
    return diffusion7(np.asarray(field).astype(np.float64), steps, c, periodic=periodic)


def himeno_fp64(p, coef, omega, sweeps):
    """himeno() in double from the same fp32 inputs (omega as the float the
    kernel uses). Returns (p after the sweeps, gosa per sweep)."""
    a = np.array(p, dtype=np.float64, copy=True)
    b = a.copy()
    cs = [np.ascontiguousarray(c, dtype=np.float64) for c in coef]
    arr = (ctypes.c_void_p * 12)(*[c.ctypes.data for c in cs])
    gosa = np.zeros(max(1, sweeps), dtype=np.float64)
    nz, ny, nx = a.shape
    port().orc_himeno_f64(nx, ny, nz, _ptr(a), _ptr(b), ctypes.cast(arr, ctypes.c_void_p),
                          float(np.float32(omega)), sweeps, _ptr(gosa))
    return (a if sweeps % 2 == 0 else b), gosa[:sweeps]


def error_norms(got, ref):
    """Max and RMS absolute error of `got` against the FP64 oracle `ref`, the
    max error relative to max |ref|, and the largest error in units of the
    last place of got's type at the reference value."""
    g = np.asarray(got, dtype=np.float64).ravel()
    r = np.asarray(ref, dtype=np.float64).ravel()
    d = np.abs(g - r)
    scale = float(np.max(np.abs(r))) if r.size else 0.0
    ulp = np.spacing(np.abs(r).astype(np.asarray(got).dtype)).astype(np.float64)
    ulp[ulp == 0] = np.finfo(np.asarray(got).dtype).tiny
    return {"max_abs_err": float(d.max()) if d.size else 0.0,
            "rms_err": float(np.sqrt(np.mean(d * d))) if d.size else 0.0,
            "max_rel_err": float(d.max() / scale) if d.size and scale > 0 else 0.0,
            "max_ulp_err": float(np.max(d / ulp)) if d.size else 0.0}


def generic_apply(desc, arrays, lo, hi, color=-1):
    """Apply a psb_generic_stencil (ctypes struct) once, in place on arrays
    (numpy, dense x-fastest, one per grid slot)."""
    ptrs = (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    dims = np.zeros(3 * len(arrays), dtype=np.int32)
    for i, a in enumerate(arrays):
        shp = list(reversed(a.shape))
        for k in range(3):
            dims[3 * i + k] = shp[k] if k < len(shp) else 1
    lo_a = np.asarray(list(lo) + [0] * (3 - len(lo)), dtype=np.int32)
    hi_a = np.asarray(list(hi) + [1] * (3 - len(hi)), dtype=np.int32)
    port().orc_generic_apply(ctypes.addressof(desc), ctypes.cast(ptrs, ctypes.c_void_p),
                             _ptr(dims), _ptr(lo_a), _ptr(hi_a), color)


def fold(op, data):
    """The reference CPU PSReduce: sequential fold from d[0] in the element type."""
    d = np.ascontiguousarray(data).ravel()
    if d.dtype == np.float32:
        out = np.zeros(1, dtype=np.float32)
        port().orc_fold_f32(op, _ptr(d), d.size, _ptr(out))
    else:
        d = d.astype(np.float64, copy=False)
        out = np.zeros(1, dtype=np.float64)
        port().orc_fold_f64(op, _ptr(d), d.size, _ptr(out))
    return out[0]


def sum_f64(data):
    """(compensated FP64 sum, sum of |x|) of a float or double array."""
    d = np.ascontiguousarray(data).ravel()
    t = PS_FLOAT if d.dtype == np.float32 else PS_DOUBLE
    if t == PS_DOUBLE:
        d = d.astype(np.float64, copy=False)
    s, a = np.zeros(1), np.zeros(1)
    port().orc_sum_f64(_ptr(d), t, d.size, _ptr(s), _ptr(a))
    return float(s[0]), float(a[0])


# ---------------------------------------------------------------------------
# Reference entry points
# ---------------------------------------------------------------------------
def ref_diffusion7(field, count, coef, periodic=False):
    """The reference CPU target: count double-buffered steps (count even).
    Returns (field, run-loop seconds)."""
    dt = field.dtype
    a = np.array(field, dtype=dt, copy=True, order="C")
    c = np.asarray(coef, dtype=dt)
    nz, ny, nx = a.shape
    f = ref().refp_diffusion7_f32 if dt == np.float32 else ref().refp_diffusion7_f64
    secs = f(nx, ny, nz, _ptr(a), count, _ptr(c), 1 if periodic else 0)
    return a, secs


def ref_himeno(p, coef, omega, nn):
    a = np.array(p, dtype=np.float32, copy=True)
    cs = [np.ascontiguousarray(c, dtype=np.float32) for c in coef]
    arr = (ctypes.c_void_p * 12)(*[c.ctypes.data for c in cs])
    nz, ny, nx = a.shape
    secs = ref().refp_himeno_f32(nx, ny, nz, _ptr(a), ctypes.cast(arr, ctypes.c_void_p),
                                 ctypes.c_float(omega), nn)
    return a, secs


def ref_box27(field, count, c):
    """The reference CPU target running the 27-point box average (count
    even double-buffered steps). Returns (field, run-loop seconds)."""
    a = np.array(field, dtype=np.float32, copy=True, order="C")
    nz, ny, nx = a.shape
    secs = ref().refp_box27_f32(nx, ny, nz, _ptr(a), count, ctypes.c_float(c))
    return a, secs


def ref_reduce(op, data):
    d = np.ascontiguousarray(data).ravel()
    if d.dtype == np.float32:
        out = np.zeros(1, dtype=np.float32)
        ref().refp_reduce_f32(op, _ptr(d), d.size, _ptr(out))
    else:
        out = np.zeros(1, dtype=np.float64)
        ref().refp_reduce_f64(op, _ptr(d), d.size, _ptr(out))
    return out[0]
