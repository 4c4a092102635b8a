"""Translator-free front end: DSL stencil functions -> sm_100a stencil kernels.

The reference turns stencil functions written in its C DSL into GPU kernels
with a ROSE-based source-to-source translator (`physisc`,
translator/cuda_translator.cc; the DSL rules are docs/programming.md:117-190).
This module does the same job without ROSE: it parses the C source with
pycparser, checks the DSL rules, rewrites the grid intrinsics into device
helpers and emits one CUDA kernel per stencil function, in the shape of the
reference's generated kernel (one thread per (x, y) point of the domain, a
loop over z, cuda_translator.cc:615-869; red-black ordering by the parity of
x+y+z, :717-727). nvcc compiles it for sm_100a into a shared library whose
launch function is registered with the runtime (psb_compiled_register), so
the kernel id works with PSStencilMap / PSStencilRun like a built-in kernel.

What is translated:
  * stencil functions: `void f(const int x[, const int y[, const int z]],
    grids..., scalars...)` with grids of type PSGrid{1,2,3}D{Float,Double,
    Int,Long} and scalars of type float, double, int or long;
  * PSGridGet(g, i, j, k) and PSGridGetPeriodic(g, ...) with integer index
    expressions (normally an index parameter plus or minus a constant; a
    lower-rank grid names the index parameters of the axes it follows);
    PSGridEmit(g, v) (stores v at the current point); PSGridDim(g, d);
  * calls to other functions of the source (stencil functions or plain C
    helpers, emitted as device functions), and C math functions;
  * any other C statement (declarations, branches, loops), as written.

Semantics kept from C: the body is emitted as C++ that evaluates the same
expressions in the same order, compiled with -fmad=false (no contraction)
and IEEE division and square root, so float arithmetic matches the
reference's CPU target bit for bit. C math functions called on float
arguments are called on (double) arguments, as C's promotion does (C++
would pick the float overloads). Every read is bounds-checked: a read
outside its grid returns 0 and sets PSB_ERR_BOUNDS, which psb_sync and
copy-out report (the reference reads out of bounds silently).
"""
import ctypes
import hashlib
import os
import re
import subprocess

from pycparser import c_ast, c_generator, c_parser

import physis_b200 as ps

HERE = os.path.dirname(os.path.abspath(__file__))
INCLUDE = os.path.join(HERE, "..", "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
DEFAULT_CACHE = os.path.join(HERE, "lib", "dsl")

_GRID_TYPES = {}
for _nd in (1, 2, 3):
    for _tn, _t in (("Float", ps.PS_FLOAT), ("Double", ps.PS_DOUBLE), ("Int", ps.PS_INT),
                    ("Long", ps.PS_LONG)):
        _GRID_TYPES["PSGrid%dD%s" % (_nd, _tn)] = (_nd, _t)
_SCALAR_TYPES = {"float": ps.PS_FLOAT, "double": ps.PS_DOUBLE, "int": ps.PS_INT,
                 "long": ps.PS_LONG}
_CTYPE = {ps.PS_FLOAT: "float", ps.PS_DOUBLE: "double", ps.PS_INT: "int",
          ps.PS_LONG: "long long"}
# C math functions whose double form C calls for float arguments.
_MATH_DOUBLE = {"sqrt", "cbrt", "sin", "cos", "tan", "asin", "acos", "atan", "atan2", "sinh",
                "cosh", "tanh", "exp", "exp2", "expm1", "log", "log2", "log10", "log1p", "pow",
                "fabs", "floor", "ceil", "round", "trunc", "fmod", "fmin", "fmax", "hypot",
                "erf", "erfc"}
_INTRINSICS = {"PSGridGet", "PSGridGetPeriodic", "PSGridEmit", "PSGridDim"}


class DSLError(ValueError):
    """The source breaks a DSL rule or cannot be translated."""


def _preprocess(source):
    """Expand the source's own macros with the C preprocessor; #include lines
    are dropped first (the DSL headers only declare what this module knows,
    and pycparser parses plain C without system headers)."""
    lines = []
    for line in source.split("\n"):
        lines.append("" if re.match(r"\s*#\s*include\b", line) else line)
    r = subprocess.run(["gcc", "-E", "-x", "c", "-"], input="\n".join(lines),
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise DSLError("the C preprocessor failed on the stencil source:\n" + r.stderr)
    return r.stdout


def _prelude():
    names = list(_GRID_TYPES) + ["PSStencil", "PSDomain1D", "PSDomain2D", "PSDomain3D",
                                 "PSIndex", "size_t", "int64_t", "int32_t", "uint64_t", "FILE"]
    return "".join("typedef int %s;\n" % n for n in names)


class _Param:
    def __init__(self, name, kind, ctype=None, nd=0):
        self.name, self.kind, self.ctype, self.nd = name, kind, ctype, nd


class StencilInfo:
    """What the front end learned about one stencil function."""

    def __init__(self, name, ndims, index_names, grids, scalars):
        self.name = name
        self.ndims = ndims
        self.index_names = index_names
        self.grids = grids          # [(name, type, nd)]
        self.scalars = scalars      # [(name, type)]
        self.emits = [0] * len(grids)
        self.reads_offset = [0] * len(grids)
        self.axes = [None] * len(grids)

    @property
    def grid_types(self):
        return [t for _, t, _ in self.grids]


def _params_of(fd):
    args = fd.decl.type.args
    out = []
    if args is None:
        return out
    for p in args.params:
        if isinstance(p, c_ast.EllipsisParam):
            raise DSLError("%s: variadic functions are not stencil functions" % fd.decl.name)
        if isinstance(p, c_ast.Typename) and isinstance(p.type, c_ast.TypeDecl) and \
                p.type.type.names == ["void"]:
            continue
        t = p.type
        if not isinstance(t, c_ast.TypeDecl) or not isinstance(t.type, c_ast.IdentifierType):
            out.append(_Param(p.name, "other"))
            continue
        tn = " ".join(t.type.names)
        if tn in _GRID_TYPES:
            nd, typ = _GRID_TYPES[tn]
            out.append(_Param(p.name, "grid", typ, nd))
        elif tn == "int" and "const" in p.quals:
            out.append(_Param(p.name, "index", ps.PS_INT))
        elif tn in _SCALAR_TYPES or tn == "long int":
            out.append(_Param(p.name, "scalar", _SCALAR_TYPES.get(tn, ps.PS_LONG)))
        else:
            out.append(_Param(p.name, "other"))
    return out


def _is_stencil(params):
    if not params or params[0].kind != "index":
        return False
    return any(p.kind == "grid" for p in params)


def _const_int(node):
    if isinstance(node, c_ast.Constant) and node.type == "int":
        return int(node.value.rstrip("uUlL"), 0)
    if isinstance(node, c_ast.UnaryOp) and node.op == "-":
        v = _const_int(node.expr)
        return None if v is None else -v
    return None


def _index_form(node, index_names):
    """(axis, offset) of an `x`, `x + c` or `x - c` index expression."""
    if isinstance(node, c_ast.ID) and node.name in index_names:
        return index_names.index(node.name), 0
    if isinstance(node, c_ast.BinaryOp) and node.op in "+-" and isinstance(node.left, c_ast.ID) \
            and node.left.name in index_names:
        c = _const_int(node.right)
        if c is not None:
            return index_names.index(node.left.name), c if node.op == "+" else -c
    return None


class _Rewriter:
    """Rewrites the intrinsics of one function body in place."""

    def __init__(self, fname, params, info, functions):
        self.fname = fname
        self.index_names = [p.name for p in params if p.kind == "index"]
        self.grids = {p.name: (i, p) for i, p in enumerate(p for p in params if p.kind == "grid")}
        self.info = info
        self.functions = functions

    def fail(self, node, msg):
        where = ""
        if getattr(node, "coord", None) is not None:
            where = " (line %d)" % node.coord.line
        raise DSLError("%s%s: %s" % (self.fname, where, msg))

    def grid_arg(self, call, node):
        if not isinstance(node, c_ast.ID) or node.name not in self.grids:
            self.fail(call, "the first argument of %s must be a grid parameter" % call.name.name)
        return self.grids[node.name]

    def visit(self, node):
        for name, child in list(node.children()):
            new = self.visit(child)
            if new is not child:
                m = re.match(r"(\w+)\[(\d+)\]$", name)
                if m:
                    getattr(node, m.group(1))[int(m.group(2))] = new
                else:
                    setattr(node, name, new)
        if isinstance(node, c_ast.FuncCall) and isinstance(node.name, c_ast.ID):
            return self.call(node)
        if isinstance(node, c_ast.UnaryOp) and node.op == "&" and isinstance(node.expr, c_ast.ID) \
                and node.expr.name in self.grids:
            self.fail(node, "taking the address of a grid is not allowed")
        return node

    def call(self, node):
        fn = node.name.name
        args = node.args.exprs if node.args else []
        if fn in ("PSGridGet", "PSGridGetPeriodic"):
            slot, p = self.grid_arg(node, args[0] if args else None)
            idx = args[1:]
            if len(idx) != p.nd:
                self.fail(node, "%s of a %d-D grid takes %d indices" % (fn, p.nd, p.nd))
            # The reference's translator wants `index parameter +- constant`
            # (for its halo analysis, docs/programming.md:161-171); here any
            # integer expression is read (reads are bounds-checked), and a
            # read that is not at the point itself marks the grid as read
            # off the point (no in-place update without red-black order).
            forms = [_index_form(e, self.index_names) for e in idx]
            at_point = len(idx) == len(self.index_names) and all(
                f is not None and f == (k, 0) for k, f in enumerate(forms))
            if self.info is not None:
                if not at_point:
                    self.info.reads_offset[slot] = 1
                if all(f is not None for f in forms):
                    axes = [f[0] for f in forms]
                    if self.info.axes[slot] is None:
                        self.info.axes[slot] = axes
            helper = "__psb_getp" if fn == "PSGridGetPeriodic" else "__psb_get"
            return c_ast.FuncCall(c_ast.ID(helper), c_ast.ExprList([c_ast.ID(p.name)] + idx),
                                  node.coord)
        if fn == "PSGridEmit":
            if len(args) != 2:
                self.fail(node, "PSGridEmit takes a grid and a value")
            slot, p = self.grid_arg(node, args[0])
            if p.nd != len(self.index_names):
                self.fail(node, "PSGridEmit into a %d-D grid from a %d-D stencil" %
                          (p.nd, len(self.index_names)))
            if self.info is not None:
                self.info.emits[slot] = 1
            pos = [c_ast.ID(n) for n in self.index_names]
            return c_ast.FuncCall(c_ast.ID("__psb_emit"),
                                  c_ast.ExprList([c_ast.ID(p.name)] + pos + [args[1]]), node.coord)
        if fn == "PSGridDim":
            if len(args) != 2:
                self.fail(node, "PSGridDim takes a grid and a dimension")
            self.grid_arg(node, args[0])
            return c_ast.FuncCall(c_ast.ID("__psb_dim"), c_ast.ExprList(list(args)), node.coord)
        if fn.startswith("PS"):
            self.fail(node, "%s is not available inside a stencil function" % fn)
        if fn in _MATH_DOUBLE and fn not in self.functions:
            dargs = [c_ast.Cast(c_ast.Typename(None, [], None, c_ast.TypeDecl(
                None, [], None, c_ast.IdentifierType(["double"]))), a) for a in args]
            return c_ast.FuncCall(c_ast.ID(fn), c_ast.ExprList(dargs), node.coord)
        return node


_HELPERS = r"""
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include "physis_b200.h"

template <typename T>
struct __psb_grid {
  T *p;
  long long sy, sz;
  int n0, n1, n2;
  int *err;
};

template <typename T>
__device__ __forceinline__ __psb_grid<T> __psb_bind(const psb_grid_view &v, int *err) {
  __psb_grid<T> g;
  g.p = (T *)v.origin;
  g.sy = v.sy;
  g.sz = v.sz;
  g.n0 = v.n[0];
  g.n1 = v.n[1];
  g.n2 = v.n[2];
  g.err = err;
  return g;
}

template <typename T>
__device__ __forceinline__ T __psb_get(const __psb_grid<T> &g, int i, int j = 0, int k = 0) {
  if ((unsigned)i >= (unsigned)g.n0 || (unsigned)j >= (unsigned)g.n1 ||
      (unsigned)k >= (unsigned)g.n2) {
    atomicExch(g.err, (int)PSB_ERR_BOUNDS);
    return T(0);
  }
  return g.p[i + j * g.sy + k * g.sz];
}

__device__ __forceinline__ int __psb_wrap(int i, int n) { return ((i % n) + n) % n; }

template <typename T>
__device__ __forceinline__ T __psb_getp(const __psb_grid<T> &g, int i, int j = 0, int k = 0) {
  return g.p[__psb_wrap(i, g.n0) + __psb_wrap(j, g.n1) * g.sy + __psb_wrap(k, g.n2) * g.sz];
}

template <typename T, typename V>
__device__ __forceinline__ void __psb_emit(const __psb_grid<T> &g, int i, V v) {
  g.p[i] = (T)v;
}
template <typename T, typename V>
__device__ __forceinline__ void __psb_emit(const __psb_grid<T> &g, int i, int j, V v) {
  g.p[i + j * g.sy] = (T)v;
}
template <typename T, typename V>
__device__ __forceinline__ void __psb_emit(const __psb_grid<T> &g, int i, int j, int k, V v) {
  g.p[i + j * g.sy + k * g.sz] = (T)v;
}

template <typename T>
__device__ __forceinline__ int __psb_dim(const __psb_grid<T> &g, int d) {
  return d == 0 ? g.n0 : (d == 1 ? g.n1 : g.n2);
}
"""


def _signature(fname, params):
    out = []
    for p in params:
        if p.kind == "index":
            out.append("const int %s" % p.name)
        elif p.kind == "grid":
            out.append("const __psb_grid<%s> %s" % (_CTYPE[p.ctype], p.name))
        elif p.kind == "scalar":
            out.append("%s %s" % (_CTYPE[p.ctype], p.name))
    return "__device__ void %s(%s)" % (fname, ", ".join(out))


class _Calls(c_ast.NodeVisitor):
    def __init__(self):
        self.names = set()

    def visit_FuncCall(self, node):
        if isinstance(node.name, c_ast.ID):
            self.names.add(node.name.name)
        self.generic_visit(node)


def _reachable(funcs):
    """The stencil functions and the functions they call (directly or not),
    in source order; the rest of the program (main, I/O) is host code."""
    by_name = {f.decl.name: f for f in funcs}
    todo = [f.decl.name for f in funcs if _is_stencil(_params_of(f))]
    keep = set()
    while todo:
        n = todo.pop()
        if n in keep or n not in by_name:
            continue
        keep.add(n)
        v = _Calls()
        v.visit(by_name[n].body)
        todo.extend(v.names)
    return [f for f in funcs if f.decl.name in keep]


def translate(source):
    """Translate every stencil function of `source`.

    Returns (cuda_source, {name: StencilInfo}). Runs on the CPU only."""
    text = _prelude() + _preprocess(source)
    try:
        ast = c_parser.CParser().parse(text, filename="<dsl>")
    except Exception as e:  # pycparser raises ParseError with a location
        raise DSLError("cannot parse the stencil source: %s" % e) from None
    gen = c_generator.CGenerator()
    funcs = [n for n in ast.ext if isinstance(n, c_ast.FuncDef)]
    names = {f.decl.name for f in funcs}
    funcs = _reachable(funcs)
    infos = {}
    parts = [_HELPERS]
    # Declarations first, so functions may call each other in any order.
    decls = []
    bodies = []
    for fd in funcs:
        fname = fd.decl.name
        if fname == "main":
            continue
        params = _params_of(fd)
        if _is_stencil(params):
            ret = fd.decl.type.type
            if not (isinstance(ret, c_ast.TypeDecl) and ret.type.names == ["void"]):
                raise DSLError("%s: stencil functions return void" % fname)
            kinds = [p.kind for p in params]
            nidx = 0
            while nidx < len(kinds) and kinds[nidx] == "index":
                nidx += 1
            if nidx > 3 or any(k == "index" for k in kinds[nidx:]):
                raise DSLError("%s: 1 to 3 `const int` index parameters come first" % fname)
            if any(k == "other" for k in kinds):
                raise DSLError("%s: parameters must be grids or float/double/int/long scalars" %
                               fname)
            grids = [(p.name, p.ctype, p.nd) for p in params if p.kind == "grid"]
            scalars = [(p.name, p.ctype) for p in params if p.kind == "scalar"]
            if len(grids) > ps.PSB_MAX_GRIDS or len(scalars) > ps.PSB_MAX_PARAMS:
                raise DSLError("%s: too many grid or scalar parameters" % fname)
            info = StencilInfo(fname, nidx, [p.name for p in params[:nidx]], grids, scalars)
            _Rewriter(fname, params, info, names).visit(fd.body)
            for slot, (gname, _, nd) in enumerate(grids):
                if info.emits[slot] and info.axes[slot] is None:
                    info.axes[slot] = list(range(nd))
            infos[fname] = info
            sig = _signature(fname, params)
        else:
            _Rewriter(fname, params, None, names).visit(fd.body)
            sig = "__device__ " + gen.visit(fd.decl).rstrip(";")
        decls.append(sig + ";")
        bodies.append(sig + "\n" + gen.visit(fd.body))
    if not infos:
        raise DSLError("no stencil function (`void f(const int x, ..., grids, ...)`) found")
    parts.append("\n".join(decls))
    parts.append("\n\n".join(bodies))
    for info in infos.values():
        parts.append(_entry(info))
    return "\n\n".join(parts) + "\n", infos


def _entry(info):
    """The kernel, launch and describe functions of one stencil function."""
    n = info.name
    binds = []
    args = ["x", "y", "z"][:info.ndims]
    for slot, (gname, t, nd) in enumerate(info.grids):
        binds.append("  const __psb_grid<%s> g%d = __psb_bind<%s>(A.grids[%d], A.error);" %
                     (_CTYPE[t], slot, _CTYPE[t], slot))
        args.append("g%d" % slot)
    for k, (sname, t) in enumerate(info.scalars):
        args.append("(%s)A.params[%d]" % (_CTYPE[t], k))
    gt = ", ".join(str(t) for t in info.grid_types)
    gn = ", ".join(str(nd) for _, _, nd in info.grids)
    em = ", ".join(str(e) for e in info.emits)
    ro = ", ".join(str(r) for r in info.reads_offset)
    pt = ", ".join(str(t) for _, t in info.scalars) or "0"
    return """
extern "C" __global__ void __launch_bounds__(256) __psb_kernel_{n}(const psb_launch_args A) {{
  // One thread per (x, y) point of the domain, a loop over z.
  const int x = A.lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = A.lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (x >= A.hi[0] || y >= A.hi[1]) return;
{binds}
  for (int z = A.lo[2]; z < A.hi[2]; z++) {{
    if (A.color >= 0 && ((x + y + z + A.color) & 1)) continue;
    {n}({args});
  }}
}}

extern "C" psb_status psb_dsl_launch_{n}(const psb_launch_args *a, void *stream) {{
  const int ex = a->hi[0] - a->lo[0], ey = a->hi[1] - a->lo[1], ez = a->hi[2] - a->lo[2];
  if (ex <= 0 || ey <= 0 || ez <= 0) return PSB_OK;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return PSB_ERR_CUDA;
  if (dev != a->device && cudaSetDevice(a->device) != cudaSuccess) return PSB_ERR_CUDA;
  const dim3 block(64, 4);
  const dim3 grid((unsigned)((ex + 63) / 64), (unsigned)((ey + 3) / 4));
  __psb_kernel_{n}<<<grid, block, 0, (cudaStream_t)stream>>>(*a);
  return cudaGetLastError() == cudaSuccess ? PSB_OK : PSB_ERR_CUDA;
}}

extern "C" void psb_dsl_describe_{n}(psb_compiled_stencil *d) {{
  const int gt[] = {{{gt}}}, gn[] = {{{gn}}}, em[] = {{{em}}}, ro[] = {{{ro}}}, pt[] = {{{pt}}};
  d->ndims = {nd};
  d->ngrids = {ng};
  for (int i = 0; i < {ng}; i++) {{
    d->grid_type[i] = gt[i];
    d->grid_ndims[i] = gn[i];
    d->emits[i] = em[i];
    d->reads_offset[i] = ro[i];
  }}
  d->nparams = {np};
  for (int i = 0; i < {np}; i++) d->param_type[i] = pt[i];
  d->launch = psb_dsl_launch_{n};
}}
""".format(n=n, binds="\n".join(binds), args=", ".join(args), gt=gt, gn=gn, em=em, ro=ro, pt=pt,
           nd=info.ndims, ng=len(info.grids), np=len(info.scalars))


def build_library(cuda_source, cache_dir=None):
    """Compile generated source for sm_100a into a shared library (cached by
    the hash of the source); returns its path."""
    cache_dir = cache_dir or DEFAULT_CACHE
    os.makedirs(cache_dir, exist_ok=True)
    key = hashlib.sha256(cuda_source.encode()).hexdigest()[:20]
    so = os.path.join(cache_dir, "libpsb_dsl_%s.so" % key)
    if os.path.exists(so):
        return so
    cu = os.path.join(cache_dir, "psb_dsl_%s.cu" % key)
    with open(cu, "w") as f:
        f.write(cuda_source)
    tmp = so + ".tmp%d" % os.getpid()
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-fmad=false", "-Xcompiler", "-fPIC", "-shared", "-I" + INCLUDE, cu, "-o", tmp]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise DSLError("nvcc failed on the generated kernel:\n" + r.stdout + r.stderr)
    os.replace(tmp, so)
    return so


_LIBS = []  # loaded kernel libraries stay loaded while registered


class CompiledStencil:
    """A stencil function compiled and registered; `kernel_id` goes to
    PSStencilMap like a built-in kernel."""

    def __init__(self, info, kernel_id, library):
        self.info = info
        self.kernel_id = kernel_id
        self.library = library

    @property
    def name(self):
        return self.info.name


def compile_stencils(source, cache_dir=None):
    """Translate, compile and register every stencil function of `source`;
    returns {name: CompiledStencil}."""
    cuda_source, infos = translate(source)
    so = build_library(cuda_source, cache_dir)
    lib = ctypes.CDLL(so)
    _LIBS.append(lib)
    out = {}
    for name, info in infos.items():
        desc = ps.CompiledStencilStruct()
        getattr(lib, "psb_dsl_describe_" + name)(ctypes.byref(desc))
        kid = ctypes.c_int()
        ps.check(ps.lib.psb_compiled_register(ctypes.byref(desc), ctypes.byref(kid)),
                 "psb_compiled_register")
        ps._generic_arity[kid.value] = len(info.grids)
        out[name] = CompiledStencil(info, kid.value, so)
    return out


def main(argv=None):
    """physis-b200-dsl: translate a DSL source into generated CUDA or a
    compiled kernel library (for C programs, which register the kernels with
    psb_dsl_describe_<name> and psb_compiled_register)."""
    import argparse
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("source")
    ap.add_argument("-o", "--output", required=True,
                    help="output: a .cu file (translation only) or a .so file")
    args = ap.parse_args(argv)
    with open(args.source) as f:
        cuda_source, infos = translate(f.read())
    if args.output.endswith(".cu"):
        with open(args.output, "w") as f:
            f.write(cuda_source)
    else:
        so = build_library(cuda_source, os.path.dirname(os.path.abspath(args.output)))
        os.replace(so, args.output)
    for name, info in infos.items():
        print("%s: %d-D, grids %s, scalars %s" % (name, info.ndims,
                                                  [g for g, _, _ in info.grids],
                                                  [s for s, _ in info.scalars]))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
