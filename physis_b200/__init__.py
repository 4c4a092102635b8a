"""physis_b200 -- Python mirror of the Physis stencil API over the B200 runtime.

The product is the C-ABI library ``lib/libphysis_rt_b200.so`` (declared in
``include/physis_b200.h``). This module binds it with ctypes and exposes the
reference's user-facing names (include/physis/physis_user.h,
include/physis/physis_common.h) so programs and tests read like the
reference's own:

    import physis_b200 as ps
    ps.PSInit()
    g1 = ps.PSGrid3DFloatNew(nx, ny, nz)
    ps.PSGridCopyin(g1, field)
    dom = ps.PSDomain3DNew(0, nx, 0, ny, 0, nz)
    m1 = ps.PSStencilMap(ps.DIFFUSION7, dom, g1, g2, ce, cw, cn, cs, ct, cb, cc)
    m2 = ps.PSStencilMap(ps.DIFFUSION7, dom, g2, g1, ce, cw, cn, cs, ct, cb, cc)
    ps.PSStencilRun(m1, m2, count // 2)
    out = ps.PSGridCopyout(g1)
    total = ps.PSReduce(ps.PS_SUM, g1)

There is no CPU fallback: importing this module without the built library
raises ImportError, and every call runs on the GPU.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# PHYSIS_B200_LIB selects another build of the library (same ABI).
LIB_PATH = os.environ.get("PHYSIS_B200_LIB") or os.path.join(_HERE, "lib", "libphysis_rt_b200.so")

# ---------------------------------------------------------------------------
# Constants (include/physis_b200.h)
# ---------------------------------------------------------------------------
PS_INT, PS_LONG, PS_FLOAT, PS_DOUBLE = 0, 1, 2, 3
PS_MAX, PS_MIN, PS_SUM, PS_PROD = 0, 1, 2, 3
PSB_HALO = 2
PSB_MAX_GRIDS = 16
PSB_MAX_TERMS = 32
PSB_MAX_PARAMS = 16
LAYOUT_DENSE, LAYOUT_PITCHED = 0, 1
DIFFUSION7, DIFFUSION7_PERIODIC, HIMENO19 = 1, 2, 3
BOUNDARY_NONE, BOUNDARY_PERIODIC, BOUNDARY_CLAMP = 0, 1, 2
IMPL_AUTO, IMPL_PLAIN, IMPL_TMA, IMPL_GENERIC = 0, 1, 2, 3
STATUS = {0: "ok", 1: "invalid argument", 2: "out of device memory or budget", 3: "CUDA error",
          4: "runtime not initialised", 5: "device-side wait timed out", 6: "unsupported",
          7: "cancelled", 8: "busy", 9: "read outside the grid"}
PSB_OK, PSB_ERR_INVALID, PSB_ERR_NOMEM, PSB_ERR_CUDA = 0, 1, 2, 3
PSB_ERR_NOT_INIT, PSB_ERR_TIMEOUT, PSB_ERR_UNSUPPORTED, PSB_ERR_CANCELLED, PSB_ERR_BUSY = 4, 5, 6, 7, 8
PSB_ERR_BOUNDS = 9

NP_TYPE = {PS_FLOAT: np.float32, PS_DOUBLE: np.float64, PS_INT: np.int32, PS_LONG: np.int64}


class PhysisError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__("%s: %s (%d)" % (what, STATUS.get(status, "?"), status))


# ---------------------------------------------------------------------------
# ctypes mirrors of the ABI structs
# ---------------------------------------------------------------------------
class PSGridStruct(ctypes.Structure):
    """__PSGrid (include/physis/physis_cuda.h:99-106)."""
    _fields_ = [("p0", ctypes.c_void_p), ("dim", ctypes.c_int * 3), ("elm_size", ctypes.c_int),
                ("num_dims", ctypes.c_int), ("num_elms", ctypes.c_int64),
                ("dev", ctypes.c_void_p)]


class PSDomain(ctypes.Structure):
    """__PSDomain (include/physis/physis_common.h:86-91)."""
    _fields_ = [("min", ctypes.c_int32 * 3), ("max", ctypes.c_int32 * 3),
                ("local_min", ctypes.c_int32 * 3), ("local_max", ctypes.c_int32 * 3)]


class Factor(ctypes.Structure):
    _fields_ = [("grid", ctypes.c_int), ("offset", ctypes.c_int * 3), ("boundary", ctypes.c_int),
                ("constant", ctypes.c_double)]


class Term(ctypes.Structure):
    _fields_ = [("a", Factor), ("b", Factor)]


class GenericStencilStruct(ctypes.Structure):
    _fields_ = [("ndims", ctypes.c_int), ("ngrids", ctypes.c_int),
                ("grid_type", ctypes.c_int * PSB_MAX_GRIDS),
                ("grid_axes", (ctypes.c_int * 3) * PSB_MAX_GRIDS), ("out_grid", ctypes.c_int),
                ("accum_type", ctypes.c_int), ("nterms", ctypes.c_int),
                ("terms", Term * PSB_MAX_TERMS), ("has_post", ctypes.c_int), ("post", Factor),
                ("redblack", ctypes.c_int)]


class GridViewStruct(ctypes.Structure):
    """psb_grid_view."""
    _fields_ = [("origin", ctypes.c_void_p), ("sy", ctypes.c_int64), ("sz", ctypes.c_int64),
                ("n", ctypes.c_int * 3), ("type", ctypes.c_int)]


PSB_MAX_VIEWS = 64


class LaunchArgs(ctypes.Structure):
    """psb_launch_args."""
    _fields_ = [("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3), ("color", ctypes.c_int),
                ("nviews", ctypes.c_int), ("nparams", ctypes.c_int),
                ("views", GridViewStruct * PSB_MAX_VIEWS),
                ("params", ctypes.c_double * PSB_MAX_PARAMS), ("error", ctypes.c_void_p),
                ("device", ctypes.c_int)]


class CompiledStencilStruct(ctypes.Structure):
    """psb_compiled_stencil."""
    _fields_ = [("ndims", ctypes.c_int), ("ngrids", ctypes.c_int),
                ("grid_type", ctypes.c_int * PSB_MAX_GRIDS),
                ("grid_ndims", ctypes.c_int * PSB_MAX_GRIDS),
                ("grid_components", ctypes.c_int * PSB_MAX_GRIDS), ("nviews", ctypes.c_int),
                ("view_type", ctypes.c_int * PSB_MAX_VIEWS),
                ("view_emits", ctypes.c_int * PSB_MAX_VIEWS),
                ("view_reads_offset", ctypes.c_int * PSB_MAX_VIEWS), ("nparams", ctypes.c_int),
                ("param_type", ctypes.c_int * PSB_MAX_PARAMS), ("launch", ctypes.c_void_p),
                ("staged_type", ctypes.c_int), ("staged_emit", ctypes.c_int),
                ("read_lo", (ctypes.c_int * 3) * PSB_MAX_GRIDS),
                ("read_hi", (ctypes.c_int * 3) * PSB_MAX_GRIDS), ("staged", ctypes.c_void_p),
                ("staged_checked", ctypes.c_void_p),
                ("read_periodic", ctypes.c_int * PSB_MAX_GRIDS)]


class TuneConfig(ctypes.Structure):
    _fields_ = [("impl", ctypes.c_int), ("tile_x", ctypes.c_int), ("tile_y", ctypes.c_int),
                ("z_chunk", ctypes.c_int), ("stages", ctypes.c_int), ("t_depth", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


PSB_MAX_FIELDS = 16
PS_USER = 4


class UserType(ctypes.Structure):
    """psb_user_type."""
    _fields_ = [("nfields", ctypes.c_int), ("record_bytes", ctypes.c_size_t),
                ("field_type", ctypes.c_int * PSB_MAX_FIELDS),
                ("field_count", ctypes.c_int * PSB_MAX_FIELDS),
                ("field_offset", ctypes.c_size_t * PSB_MAX_FIELDS)]


class Request(ctypes.Structure):
    """psb_request."""
    _fields_ = [("kernel_id", ctypes.c_int), ("dims", ctypes.c_int32 * 3),
                ("max_steps", ctypes.c_int), ("tol", ctypes.c_double),
                ("check_every", ctypes.c_int), ("init", ctypes.c_void_p),
                ("coef", ctypes.c_void_p), ("out", ctypes.c_void_p), ("seed", ctypes.c_uint64),
                ("params", ctypes.c_double * PSB_MAX_PARAMS), ("nparams", ctypes.c_int)]


class Result(ctypes.Structure):
    """psb_result."""
    _fields_ = [("id", ctypes.c_int64), ("status", ctypes.c_int), ("steps_done", ctypes.c_int),
                ("residual", ctypes.c_double), ("submit_s", ctypes.c_double),
                ("start_s", ctypes.c_double), ("finish_s", ctypes.c_double),
                ("wave_rounds", ctypes.c_int)]


class BatchLayout(ctypes.Structure):
    """psb_batch_layout."""
    _fields_ = [("tile_x", ctypes.c_int), ("tile_y", ctypes.c_int), ("z_chunk", ctypes.c_int),
                ("tiles", ctypes.c_int), ("wavefront", ctypes.c_int), ("tuned", ctypes.c_int),
                ("t_depth", ctypes.c_int), ("units", ctypes.c_int)]


# ---------------------------------------------------------------------------
# Library loading (fails loudly; there is no fallback)
# ---------------------------------------------------------------------------
def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("physis_b200: %s is missing; run physis_b200/build.py "
                          "(or __graft_entry__.build())" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    G = ctypes.c_void_p
    S = ctypes.c_int
    sigs = {
        "PSInit": (None, [ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.c_int]),
        "PSFinalize": (None, []),
        "__PSGridNew": (G, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]),
        "__PSGridFree": (None, [G, ctypes.c_void_p]),
        "__PSGridCopyin": (None, [G, ctypes.c_void_p, ctypes.c_void_p]),
        "__PSGridCopyout": (None, [G, ctypes.c_void_p, ctypes.c_void_p]),
        "__PSGridSwap": (None, [G]),
        "__PSGridMirror": (None, [G]),
        "__PSGridGetID": (ctypes.c_int, [G]),
        "__PSReduceGridFloat": (None, [ctypes.c_void_p, ctypes.c_int, G]),
        "__PSReduceGridDouble": (None, [ctypes.c_void_p, ctypes.c_int, G]),
        "__PSCheckCudaError": (None, [ctypes.c_char_p]),
        "__PSRandomInit": (ctypes.c_void_p, [ctypes.c_int]),
        "PSGridCopyin": (None, [G, ctypes.c_void_p]),
        "PSGridCopyout": (None, [G, ctypes.c_void_p]),
        "PSGridFree": (None, [G]),
        "psb_init": (S, []),
        "PSGetLastError": (S, []),
        "psb_status_string": (ctypes.c_char_p, [S]),
        "psb_grid_new": (S, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32), ctypes.c_int,
                             ctypes.POINTER(G)]),
        "psb_grid_layout": (S, [G, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64)]),
        "psb_grid_copyin_async": (S, [G, ctypes.c_void_p]),
        "psb_grid_new_user": (S, [ctypes.c_int, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(UserType),
                                  ctypes.POINTER(G)]),
        "psb_grid_component": (S, [G, ctypes.c_int, ctypes.c_int, ctypes.POINTER(G)]),
        "psb_grid_copyout_async": (S, [G, ctypes.c_void_p]),
        "psb_sync": (S, []),
        "psb_host_alloc": (S, [ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]),
        "psb_host_free": (S, [ctypes.c_void_p]),
        "psb_grid_copy": (S, [G, G]),
        "psb_grid_fill": (S, [G, ctypes.c_int, ctypes.c_uint64, ctypes.c_double, ctypes.c_double]),
        "psb_generic_register": (S, [ctypes.POINTER(GenericStencilStruct), ctypes.POINTER(ctypes.c_int)]),
        "psb_compiled_register": (S, [ctypes.POINTER(CompiledStencilStruct),
                                      ctypes.POINTER(ctypes.c_int)]),
        "psb_stencil_map": (S, [ctypes.c_int, ctypes.POINTER(PSDomain), ctypes.POINTER(G), ctypes.c_int,
                                ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
        "psb_stencil_map_rb": (S, [ctypes.c_int, ctypes.POINTER(PSDomain), ctypes.POINTER(G), ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_int)]),
        "psb_stencil_run": (S, [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int]),
        "psb_stencil_free": (S, [ctypes.c_int]),
        "psb_set_impl": (S, [ctypes.c_int]),
        "psb_set_graph": (S, [ctypes.c_int]),
        "psb_himeno_residual_enable": (S, [ctypes.c_int, ctypes.c_int]),
        "psb_himeno_residual": (S, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
        "psb_himeno_residual_history": (S, [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int]),
        "psb_reduce": (S, [G, ctypes.c_int, ctypes.POINTER(PSDomain), ctypes.POINTER(ctypes.c_double)]),
        "psb_reduce_map": (S, [ctypes.c_int, ctypes.POINTER(PSDomain), ctypes.POINTER(G), ctypes.c_int,
                               ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                               ctypes.POINTER(ctypes.c_double)]),
        "psb_last_run_stats": (S, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]),
        "psb_autotune": (S, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32), ctypes.c_int,
                             ctypes.POINTER(TuneConfig)]),
        "psb_tune_get": (S, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                             ctypes.POINTER(TuneConfig)]),
        "psb_tune_set": (S, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                             ctypes.POINTER(TuneConfig)]),
        "psb_batch_create": (S, [ctypes.POINTER(ctypes.c_void_p)]),
        "psb_batch_add": (S, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(G), ctypes.c_int,
                              ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                              ctypes.POINTER(ctypes.c_int)]),
        "psb_batch_run": (S, [ctypes.c_void_p, ctypes.c_int]),
        "psb_batch_stats": (S, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
        "psb_batch_free": (S, [ctypes.c_void_p]),
        "psb_batch_set_stop": (S, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int]),
        "psb_batch_member_result": (S, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_int)]),
        "psb_set_fp_mode": (S, [ctypes.c_int]),
        "psb_set_generic_compile": (S, [ctypes.c_int]),
        "psb_generic_last_compiled": (S, [ctypes.POINTER(ctypes.c_int)]),
        "psb_compiled_last_staged": (S, [ctypes.POINTER(ctypes.c_int)]),
        "psb_get_fp_mode": (S, [ctypes.POINTER(ctypes.c_int)]),
        "psb_batch_member_layout": (S, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(BatchLayout)]),
        "psb_batch_autotune": (S, [ctypes.c_void_p, ctypes.c_int]),
        "psb_server_create": (S, [ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
        "psb_server_submit": (S, [ctypes.c_void_p, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_int64)]),
        "psb_server_cancel": (S, [ctypes.c_void_p, ctypes.c_int64]),
        "psb_server_wait": (S, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                                ctypes.POINTER(Result)]),
        "psb_server_request_bytes": (S, [ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_size_t)]),
        "psb_server_stats": (S, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                 ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_size_t),
                                 ctypes.POINTER(ctypes.c_double)]),
        "psb_server_destroy": (S, [ctypes.c_void_p]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    # Domain constructors return the struct by value.
    for n, k in (("PSDomain1DNew", 2), ("PSDomain2DNew", 4), ("PSDomain3DNew", 6)):
        f = getattr(lib, n)
        f.restype = PSDomain
        f.argtypes = [ctypes.c_int32] * k
    return lib


lib = _load()


def check(status, what=""):
    if status != PSB_OK:
        raise PhysisError(status, what)


# ---------------------------------------------------------------------------
# Grids
# ---------------------------------------------------------------------------
class Grid:
    """Handle of one device grid (a __PSGrid* of the runtime)."""

    def __init__(self, ptr, type_, dims):
        self.ptr = ctypes.c_void_p(ptr)
        self.type = type_
        self.dims = tuple(dims)  # (nx[, ny[, nz]]), x fastest

    @property
    def shape(self):
        """numpy shape of the dense host array: (nz, ny, nx)."""
        return tuple(reversed(self.dims))

    @property
    def dtype(self):
        return NP_TYPE[self.type]

    def layout(self):
        sy, sz, lay, nb = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int(), ctypes.c_int64()
        check(lib.psb_grid_layout(self.ptr, ctypes.byref(sy), ctypes.byref(sz), ctypes.byref(lay),
                                  ctypes.byref(nb)), "psb_grid_layout")
        return {"stride_y": sy.value, "stride_z": sz.value, "layout": lay.value,
                "alloc_bytes": nb.value}


def PSInit(argv=None):
    argv = list(argv or ["physis_b200"])
    argc = ctypes.c_int(len(argv))
    arr = (ctypes.c_char_p * (len(argv) + 1))(*[a.encode() for a in argv], None)
    parr = ctypes.pointer(arr)
    lib.PSInit(ctypes.byref(argc), ctypes.cast(ctypes.byref(parr), ctypes.c_void_p), 3)
    return [arr[i].decode() for i in range(argc.value)]


def PSFinalize():
    lib.PSFinalize()


def grid_new(type_, dims, layout=LAYOUT_PITCHED):
    d = (ctypes.c_int32 * 3)(*(list(dims) + [0] * (3 - len(dims))))
    p = ctypes.c_void_p()
    check(lib.psb_grid_new(type_, len(dims), d, layout, ctypes.byref(p)), "psb_grid_new")
    return Grid(p.value, type_, dims)


def grid_new_user(dims, fields, record_bytes):
    """Grid of a user-defined point type. fields: list of (type, count,
    byte offset) in record order; record_bytes: the record size (e.g. a
    numpy structured dtype's itemsize)."""
    ut = UserType()
    ut.nfields = len(fields)
    ut.record_bytes = int(record_bytes)
    for i, (t, n, off) in enumerate(fields):
        ut.field_type[i] = t
        ut.field_count[i] = n
        ut.field_offset[i] = off
    d = (ctypes.c_int32 * 3)(*(list(dims) + [0] * (3 - len(dims))))
    p = ctypes.c_void_p()
    check(lib.psb_grid_new_user(len(dims), d, ctypes.byref(ut), ctypes.byref(p)), "psb_grid_new_user")
    g = Grid(p.value, PS_USER, dims)
    g.fields = list(fields)
    g.record_bytes = int(record_bytes)
    return g


def component(g, field, index=0):
    """Component `index` of field `field` of a user-type grid, as a grid that
    stencils can bind (owned by g: do not free it)."""
    p = ctypes.c_void_p()
    check(lib.psb_grid_component(g.ptr, field, index, ctypes.byref(p)), "psb_grid_component")
    return Grid(p.value, g.fields[field][0], g.dims)


def user_copyin(g, records):
    """Copy a host array of records (numpy, itemsize = record_bytes) into a
    user-type grid."""
    a = np.ascontiguousarray(records)
    if a.itemsize * a.size != g.record_bytes * int(np.prod(g.dims)):
        raise ValueError("record array does not match the grid")
    check(lib.psb_grid_copyin_async(g.ptr, a.ctypes.data), "psb_grid_copyin_async")
    sync()


def user_copyout(g, records):
    """Copy a user-type grid into a host array of records (in place)."""
    if not records.flags.c_contiguous or records.itemsize * records.size != \
            g.record_bytes * int(np.prod(g.dims)):
        raise ValueError("record array does not match the grid")
    check(lib.psb_grid_copyout_async(g.ptr, records.ctypes.data), "psb_grid_copyout_async")
    sync()


def _mk(type_, nd):
    def f(*dims):
        if len(dims) != nd:
            raise TypeError("expected %d extents" % nd)
        return grid_new(type_, dims, LAYOUT_PITCHED)
    return f


PSGrid1DFloatNew, PSGrid2DFloatNew, PSGrid3DFloatNew = (_mk(PS_FLOAT, k) for k in (1, 2, 3))
PSGrid1DDoubleNew, PSGrid2DDoubleNew, PSGrid3DDoubleNew = (_mk(PS_DOUBLE, k) for k in (1, 2, 3))
PSGrid1DIntNew, PSGrid2DIntNew, PSGrid3DIntNew = (_mk(PS_INT, k) for k in (1, 2, 3))
PSGrid1DLongNew, PSGrid2DLongNew, PSGrid3DLongNew = (_mk(PS_LONG, k) for k in (1, 2, 3))


def PSGridNewDense(type_, dims):
    """A grid from the drop-in entry point __PSGridNew (dense, reference layout)."""
    esize = np.dtype(NP_TYPE[type_]).itemsize
    d = (ctypes.c_int * 3)(*(list(dims) + [0] * (3 - len(dims))))
    p = lib.__PSGridNew(esize, len(dims), d, None)
    if not p:
        raise PhysisError(PSB_ERR_NOMEM, "__PSGridNew")
    return Grid(p, type_, dims)


def PSGridCopyin(g, src):
    a = np.ascontiguousarray(src, dtype=g.dtype)
    if a.size != int(np.prod(g.dims)):
        raise ValueError("copy-in array has %d elements, grid has %d" % (a.size, np.prod(g.dims)))
    lib.PSGridCopyin(g.ptr, a.ctypes.data)


def PSGridCopyout(g, out=None):
    if out is None:
        out = np.empty(g.shape, dtype=g.dtype)
    if not out.flags.c_contiguous or out.dtype != g.dtype or out.size != int(np.prod(g.dims)):
        raise ValueError("copy-out array must be C-contiguous %s with %d elements"
                         % (g.dtype, np.prod(g.dims)))
    lib.PSGridCopyout(g.ptr, out.ctypes.data)
    return out


def PSGridFree(g):
    if g.ptr:
        lib.PSGridFree(g.ptr)
        g.ptr = ctypes.c_void_p()


FILL_UNIFORM, FILL_CONST, FILL_BND, FILL_ZPROFILE = 0, 1, 2, 3


def grid_fill(g, kind, seed=0, lo=0.0, hi=1.0):
    """Seeded synthetic field generated on the device (psb_grid_fill)."""
    check(lib.psb_grid_fill(g.ptr, kind, seed, lo, hi), "psb_grid_fill")


def fill_reference(dims, kind, seed=0, lo=0.0, hi=1.0, dtype=np.float32):
    """Host restatement of psb_grid_fill (for checks): array of shape (nz, ny, nx)."""
    nx, ny, nz = dims
    i = np.arange(nx * ny * nz, dtype=np.uint64)
    if kind == FILL_UNIFORM:
        with np.errstate(over="ignore"):
            x = np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + i + np.uint64(0x9E3779B97F4A7C15)
            x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            x = x ^ (x >> np.uint64(31))
        v = lo + (hi - lo) * ((x >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0))
    elif kind == FILL_CONST:
        v = np.full(i.shape, lo, dtype=np.float64)
    elif kind == FILL_BND:
        z, r = np.divmod(i.astype(np.int64), nx * ny)
        y, x = np.divmod(r, nx)
        face = (x == 0) | (y == 0) | (z == 0) | (x == nx - 1) | (y == ny - 1) | (z == nz - 1)
        v = np.where(face, 0.0, 1.0)
    else:
        z = i.astype(np.int64) // (nx * ny)
        t = z / (nz - 1) if nz > 1 else np.zeros_like(z, dtype=np.float64)
        v = t * t
    return v.astype(dtype).reshape(nz, ny, nx)


def PSGridDim(g, d):
    return g.dims[d]


def PSDomain1DNew(x0, x1):
    return lib.PSDomain1DNew(x0, x1)


def PSDomain2DNew(x0, x1, y0, y1):
    return lib.PSDomain2DNew(x0, x1, y0, y1)


def PSDomain3DNew(x0, x1, y0, y1, z0, z1):
    return lib.PSDomain3DNew(x0, x1, y0, y1, z0, z1)


# ---------------------------------------------------------------------------
# Stencils
# ---------------------------------------------------------------------------
class Stencil:
    """A map handle (PSStencil)."""

    def __init__(self, handle, grids):
        self.handle = handle
        self.grids = grids  # keep grids referenced

    def free(self):
        check(lib.psb_stencil_free(self.handle), "psb_stencil_free")


def _kernel_arity(kernel):
    if kernel in (DIFFUSION7, DIFFUSION7_PERIODIC):
        return 2
    if kernel == HIMENO19:
        return 14
    return _generic_arity[kernel]


_generic_arity = {}


def _map(kernel, dom, args, color):
    ng = _kernel_arity(kernel)
    grids = list(args[:ng])
    params = [float(p) for p in args[ng:]]
    gp = (ctypes.c_void_p * len(grids))(*[g.ptr.value for g in grids])
    pp = (ctypes.c_double * max(1, len(params)))(*params)
    h = ctypes.c_int()
    if color is None:
        st = lib.psb_stencil_map(kernel, ctypes.byref(dom), gp, len(grids), pp, len(params),
                                 ctypes.byref(h))
    else:
        st = lib.psb_stencil_map_rb(kernel, ctypes.byref(dom), gp, len(grids), pp, len(params),
                                    color, ctypes.byref(h))
    check(st, "PSStencilMap")
    return Stencil(h.value, grids)


def PSStencilMap(kernel, dom, *args):
    return _map(kernel, dom, args, None)


def PSStencilMapRedBlack(kernel, dom, *args):
    return _map(kernel, dom, args, 2)


def PSStencilMapRed(kernel, dom, *args):
    return _map(kernel, dom, args, 0)


def PSStencilMapBlack(kernel, dom, *args):
    return _map(kernel, dom, args, 1)


def PSStencilRun(*args):
    """PSStencilRun(m0, m1, ..., [iter]) -- maps in order, iter times."""
    iters = 1
    if args and not isinstance(args[-1], Stencil):
        iters = int(args[-1])
        args = args[:-1]
    hs = (ctypes.c_int * len(args))(*[m.handle for m in args])
    check(lib.psb_stencil_run(hs, len(args), iters), "PSStencilRun")


def last_run_stats():
    ms, n = ctypes.c_double(), ctypes.c_int64()
    check(lib.psb_last_run_stats(ctypes.byref(ms), ctypes.byref(n)), "psb_last_run_stats")
    return ms.value, n.value


def PSReduce(op, g, dom=None):
    """Reduce a grid. Returns the value in the grid's element type (as the
    reference does); psb_reduce gives the FP64 accumulator."""
    if dom is None and g.type in (PS_FLOAT, PS_DOUBLE):
        if g.type == PS_FLOAT:
            v = ctypes.c_float()
            lib.__PSReduceGridFloat(ctypes.byref(v), op, g.ptr)
        else:
            v = ctypes.c_double()
            lib.__PSReduceGridDouble(ctypes.byref(v), op, g.ptr)
        return v.value
    return reduce64(op, g, dom)


def PSReduceMap(op, kernel, dom, *grids):
    """Kernel-function reduction (the PSReduce(&v, op, kernel, dom, ...) form):
    reduce over dom the values the generic stencil `kernel` would emit with
    these grids, without storing them. Returns the FP64 result."""
    gp = (ctypes.c_void_p * len(grids))(*[g.ptr.value for g in grids])
    r = ctypes.c_double()
    check(lib.psb_reduce_map(int(kernel), ctypes.byref(dom), gp, len(grids), None, 0, op,
                             ctypes.byref(r)), "psb_reduce_map")
    return r.value


def reduce64(op, g, dom=None):
    r = ctypes.c_double()
    check(lib.psb_reduce(g.ptr, op, ctypes.byref(dom) if dom is not None else None,
                         ctypes.byref(r)), "psb_reduce")
    return r.value


def set_impl(impl):
    check(lib.psb_set_impl(impl), "psb_set_impl")


FP_EXACT, FP_FMA = 0, 1


def set_fp_mode(mode):
    """Arithmetic of the 7-point TMA kernels: FP_EXACT (the reference's
    roundings, default) or FP_FMA (fused multiply-adds, within 4 ulp)."""
    check(lib.psb_set_fp_mode(mode), "psb_set_fp_mode")


def get_fp_mode():
    m = ctypes.c_int()
    check(lib.psb_get_fp_mode(ctypes.byref(m)), "psb_get_fp_mode")
    return m.value


def set_generic_compile(on):
    """Run-time compilation of generic tables on the TMA path (default on)."""
    check(lib.psb_set_generic_compile(1 if on else 0), "psb_set_generic_compile")


def compiled_last_staged():
    """Which form the last application of a compiled (DSL) stencil ran: 0 its
    own thread-per-point launch, 1 the staged (TMA plane ring) form, 2 the
    staged form with its reads checked against their grids."""
    v = ctypes.c_int()
    check(lib.psb_compiled_last_staged(ctypes.byref(v)), "psb_compiled_last_staged")
    return v.value


def generic_last_compiled():
    """Whether the last TMA application of a generic stencil ran a kernel
    compiled for its table."""
    v = ctypes.c_int()
    check(lib.psb_generic_last_compiled(ctypes.byref(v)), "psb_generic_last_compiled")
    return bool(v.value)


def set_graph(enable):
    check(lib.psb_set_graph(1 if enable else 0), "psb_set_graph")


def sync():
    check(lib.psb_sync(), "psb_sync")


def autotune(kernel, type_, dims, force=False):
    d = (ctypes.c_int32 * 3)(*dims)
    c = TuneConfig()
    check(lib.psb_autotune(kernel, type_, d, 1 if force else 0, ctypes.byref(c)), "psb_autotune")
    return c.as_dict()


def tune_get(kernel, type_, dims):
    d = (ctypes.c_int32 * 3)(*dims)
    c = TuneConfig()
    check(lib.psb_tune_get(kernel, type_, d, ctypes.byref(c)), "psb_tune_get")
    return c.as_dict()


def tune_set(kernel, type_, dims, **cfg):
    d = (ctypes.c_int32 * 3)(*dims)
    c = TuneConfig(**cfg)
    check(lib.psb_tune_set(kernel, type_, d, ctypes.byref(c)), "psb_tune_set")


PSB_BATCH_TUNE_BASE = 100


def batch_bucket(dims):
    """Size bucket of a batch member: each extent rounded up to a power of
    two, at least 8."""
    out = []
    for n in dims:
        b = 8
        while b < n:
            b <<= 1
        out.append(b)
    return out


def batch_tune_set(kernel, dims, **cfg):
    """Pin the shape of the batch members of stencil `kernel` whose size
    bucket is that of `dims` (the PSB_BATCH_TUNE_BASE entry)."""
    tune_set(PSB_BATCH_TUNE_BASE + kernel - 1, PS_FLOAT, batch_bucket(dims), **cfg)


def himeno_residual_enable(m, history=1):
    check(lib.psb_himeno_residual_enable(m.handle, history), "psb_himeno_residual_enable")


def himeno_residual_history(m, n):
    out = (ctypes.c_double * n)()
    check(lib.psb_himeno_residual_history(m.handle, out, n), "psb_himeno_residual_history")
    return list(out)


# ---------------------------------------------------------------------------
# Generic stencils
# ---------------------------------------------------------------------------
def get(grid, offset=(0, 0, 0), boundary=BOUNDARY_NONE):
    """A grid-read factor: grid slot, offset in domain axes, boundary form."""
    return ("g", int(grid), tuple(offset) + (0,) * (3 - len(offset)), int(boundary))


def const(value):
    return ("c", float(value))


def _factor(f):
    out = Factor()
    if f[0] == "c":
        out.grid = -1
        out.constant = f[1]
    else:
        out.grid = f[1]
        for i in range(3):
            out.offset[i] = f[2][i]
        out.boundary = f[3]
    return out


def generic_struct(ndims, grids, out, accum, terms, post=None):
    """Build the psb_generic_stencil struct of a flat linear stencil.

    grids: list of (type, axes) per slot, axes = domain axis of each grid
    dimension (e.g. (0, 1, 2) for a 3-D grid, (0,) for a 1-D grid along x).
    terms: list of (factor_a, factor_b) built with get()/const(); a single
    factor means b = const(1). post: optional factor multiplied last.
    """
    s = GenericStencilStruct()
    s.ndims = ndims
    s.ngrids = len(grids)
    for i, (t, axes) in enumerate(grids):
        s.grid_type[i] = t
        ax = list(axes) + [-1] * (3 - len(axes))
        for k in range(3):
            s.grid_axes[i][k] = ax[k]
    s.out_grid = out
    s.accum_type = accum
    s.nterms = len(terms)
    for i, t in enumerate(terms):
        if isinstance(t[0], str):
            t = (t, const(1.0))
        s.terms[i].a = _factor(t[0])
        s.terms[i].b = _factor(t[1])
    if post is not None:
        s.has_post = 1
        s.post = _factor(post)
    return s


class GenericStencil:
    """A registered generic stencil; .kernel_id goes to PSStencilMap."""

    def __init__(self, ndims, grids, out, accum, terms, post=None):
        self.struct = generic_struct(ndims, grids, out, accum, terms, post)
        kid = ctypes.c_int()
        check(lib.psb_generic_register(ctypes.byref(self.struct), ctypes.byref(kid)),
              "psb_generic_register")
        self.kernel_id = kid.value
        _generic_arity[self.kernel_id] = len(grids)


# ---------------------------------------------------------------------------
# Batching
# ---------------------------------------------------------------------------
BATCH_PERSISTENT, BATCH_GRAPH, BATCH_PLAIN_LOOP, BATCH_TUNED_LOOP = 0, 1, 2, 3


class Batch:
    """Many independent solves advanced together (psb_batch_*)."""

    def __init__(self):
        p = ctypes.c_void_p()
        check(lib.psb_batch_create(ctypes.byref(p)), "psb_batch_create")
        self.ptr = p
        self.members = []

    def add(self, kernel, grids, params, steps, tol=0.0, check_every=0):
        gp = (ctypes.c_void_p * len(grids))(*[g.ptr.value for g in grids])
        pp = (ctypes.c_double * max(1, len(params)))(*[float(v) for v in params])
        m = ctypes.c_int()
        check(lib.psb_batch_add(self.ptr, kernel, gp, len(grids), pp, len(params), steps,
                                ctypes.byref(m)), "psb_batch_add")
        if tol > 0 or check_every > 0:
            check(lib.psb_batch_set_stop(self.ptr, m.value, tol, check_every), "psb_batch_set_stop")
        self.members.append(list(grids))
        return m.value

    def run(self, mode=BATCH_PERSISTENT):
        check(lib.psb_batch_run(self.ptr, mode), "psb_batch_run")

    def stats(self):
        ms, n, lups = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64()
        check(lib.psb_batch_stats(self.ptr, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(lups)),
              "psb_batch_stats")
        return {"device_ms": ms.value, "launches": n.value, "lattice_updates": lups.value}

    def result(self, member):
        """(steps done, residual, grid holding the result)."""
        st, res, which = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        check(lib.psb_batch_member_result(self.ptr, member, ctypes.byref(st), ctypes.byref(res),
                                          ctypes.byref(which)), "psb_batch_member_result")
        return st.value, res.value, self.members[member][which.value]

    def autotune(self, force=False):
        """Tune the tile shape and z chunk of every member size bucket without
        a cached entry (psb_batch_autotune)."""
        check(lib.psb_batch_autotune(self.ptr, 1 if force else 0), "psb_batch_autotune")

    def layout(self, member):
        """How the last mode-0/1 run cut the member into items (dict of
        psb_batch_layout)."""
        lay = BatchLayout()
        check(lib.psb_batch_member_layout(self.ptr, member, ctypes.byref(lay)),
              "psb_batch_member_layout")
        return {k: getattr(lay, k) for k, _ in lay._fields_}

    def tuned(self, member):
        """Whether the member's tile shape came from the autotuner's table."""
        return bool(self.layout(member)["tuned"])

    def free(self):
        if self.ptr:
            check(lib.psb_batch_free(self.ptr), "psb_batch_free")
            self.ptr = ctypes.c_void_p()


# ---------------------------------------------------------------------------
# Serving
# ---------------------------------------------------------------------------
SERVE_BATCHED = 0
SERVE_FIFO = 1


def _host_ptr(a, n, what):
    """Address of a C-contiguous float32 array of n elements (None -> NULL)."""
    if a is None:
        return None
    if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous
            and a.size == n):
        raise ValueError("%s: need a C-contiguous float32 array of %d elements" % (what, n))
    return a.ctypes.data


class Server:
    """Continuous-batching solve server (psb_server_*).

    Arrays passed to submit (init, coef, out) must stay alive until wait()
    has returned that request; the object keeps references to them until
    then."""

    def __init__(self, budget_bytes, max_slots=0, mode=SERVE_BATCHED):
        p = ctypes.c_void_p()
        check(lib.psb_server_create(int(budget_bytes), int(max_slots), int(mode), ctypes.byref(p)),
              "psb_server_create")
        self.ptr = p
        self._keep = {}

    @staticmethod
    def request(kernel, dims, params, max_steps, tol=0.0, check_every=0, init=None, coef=None,
                out=None, seed=0):
        q = Request()
        q.kernel_id = int(kernel)
        for k in range(3):
            q.dims[k] = int(dims[k])
        q.max_steps = int(max_steps)
        q.tol = float(tol)
        q.check_every = int(check_every)
        n = int(dims[0]) * int(dims[1]) * int(dims[2])
        q.init = _host_ptr(init, n, "init")
        q.coef = _host_ptr(coef, 12 * n, "coef")
        q.out = _host_ptr(out, n, "out")
        q.seed = int(seed)
        for i, v in enumerate(params):
            q.params[i] = float(v)
        q.nparams = len(params)
        return q

    @staticmethod
    def request_bytes(q):
        b = ctypes.c_size_t()
        check(lib.psb_server_request_bytes(ctypes.byref(q), ctypes.byref(b)), "psb_server_request_bytes")
        return b.value

    def submit(self, kernel, dims, params, max_steps, tol=0.0, check_every=0, init=None,
               coef=None, out=None, seed=0):
        q = self.request(kernel, dims, params, max_steps, tol, check_every, init, coef, out, seed)
        i = ctypes.c_int64()
        check(lib.psb_server_submit(self.ptr, ctypes.byref(q), ctypes.byref(i)), "psb_server_submit")
        self._keep[i.value] = (init, coef, out)
        return i.value

    def cancel(self, rid):
        check(lib.psb_server_cancel(self.ptr, int(rid)), "psb_server_cancel")

    def wait(self, rid=-1, timeout=-1.0):
        """Record of request rid (-1: the next completed one) as a dict."""
        r = Result()
        check(lib.psb_server_wait(self.ptr, int(rid), float(timeout), ctypes.byref(r)),
              "psb_server_wait")
        self._keep.pop(r.id, None)
        return {"id": r.id, "status": r.status, "steps_done": r.steps_done,
                "residual": r.residual, "submit_s": r.submit_s, "start_s": r.start_s,
                "finish_s": r.finish_s, "wave_rounds": r.wave_rounds}

    def stats(self):
        c, rd, la = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        pk, ms = ctypes.c_size_t(), ctypes.c_double()
        check(lib.psb_server_stats(self.ptr, ctypes.byref(c), ctypes.byref(rd), ctypes.byref(la),
                                   ctypes.byref(pk), ctypes.byref(ms)), "psb_server_stats")
        return {"completed": c.value, "rounds": rd.value, "launches": la.value,
                "peak_bytes": pk.value, "device_ms": ms.value}

    def destroy(self):
        if self.ptr:
            check(lib.psb_server_destroy(self.ptr), "psb_server_destroy")
            self.ptr = ctypes.c_void_p()
            self._keep.clear()
