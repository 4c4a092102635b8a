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
  * grids of user-defined point types (`struct T {...}; DeclareGrid3D(Name,
    struct T)`, members float/double/int/long scalars or fixed arrays):
    PSGridGet(g, ...).member[i][j] reads one component, PSGridGet(g, ...) the
    whole record, PSGridEmit(g, record) stores every member and
    PSGridEmitUtype(g.member[i][j], v) one (translator/cuda_runtime_builder.cc
    :319-1100 of the reference); on the device each component is its own
    grid, so a stencil may update one member of a grid in place while
    reading others around the point;
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
import threading

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


class DSLError(ValueError):
    """The source breaks a DSL rule or cannot be translated."""


_DECLARE = re.compile(r"\bDeclareGrid([123])D\s*\(\s*(\w+)\s*,\s*struct\s+(\w+)\s*\)\s*;?")


def _preprocess(source):
    """Expand the source's own macros with the C preprocessor; #include lines
    are dropped first (the DSL headers only declare what this module knows,
    and pycparser parses plain C without system headers). Grid types of
    user-defined point types, `DeclareGrid3D(Name, struct T)`, become
    typedefs; returns (text, {grid type name: (rank, struct name)})."""
    lines = []
    for line in source.split("\n"):
        lines.append("" if re.match(r"\s*#\s*include\b", line) else line)
    r = subprocess.run(["gcc", "-E", "-x", "c", "-"], input="\n".join(lines),
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise DSLError("the C preprocessor failed on the stencil source:\n" + r.stderr)
    user = {}

    def declare(m):
        user["PSGrid%sD%s" % (m.group(1), m.group(2))] = (int(m.group(1)), m.group(3))
        return "typedef int PSGrid%sD%s;" % (m.group(1), m.group(2))

    return _DECLARE.sub(declare, r.stdout), user


def _prelude():
    names = list(_GRID_TYPES) + ["PSStencil", "PSDomain1D", "PSDomain2D", "PSDomain3D",
                                 "PSIndex", "size_t", "int64_t", "int32_t", "uint64_t", "FILE"]
    return "".join("typedef int %s;\n" % n for n in names)


class _Field:
    def __init__(self, name, ctype, dims, first):
        self.name, self.ctype, self.dims, self.first = name, ctype, dims, first

    @property
    def count(self):
        n = 1
        for d in self.dims:
            n *= d
        return n


class _Struct:
    """A point type: its scalar fields (arrays flattened row-major) in order."""

    def __init__(self, name, fields):
        self.name = name
        self.fields = fields
        self.count = sum(f.count for f in fields)

    def field(self, name):
        for f in self.fields:
            if f.name == name:
                return f
        return None


def _struct_defs(ast):
    """Point types defined at file scope: struct name -> _Struct (only those
    whose members are float/double/int/long scalars or arrays of them)."""
    out = {}
    for n in ast.ext:
        t = getattr(n, "type", None)
        if isinstance(n, c_ast.Decl) and isinstance(t, c_ast.Struct) and t.decls:
            fields, first, ok = [], 0, True
            for d in t.decls:
                ty, dims = d.type, []
                while isinstance(ty, c_ast.ArrayDecl):
                    c = _const_int(ty.dim) if ty.dim is not None else None
                    if c is None or c <= 0:
                        ok = False
                        break
                    dims.append(c)
                    ty = ty.type
                if not ok or not isinstance(ty, c_ast.TypeDecl) or \
                        not isinstance(ty.type, c_ast.IdentifierType):
                    ok = False
                    break
                tn = " ".join(ty.type.names)
                if tn not in _SCALAR_TYPES and tn != "long int":
                    ok = False
                    break
                f = _Field(d.name, _SCALAR_TYPES.get(tn, ps.PS_LONG), dims, first)
                fields.append(f)
                first += f.count
            if ok:
                out[t.name] = _Struct(t.name, fields)
    return out


class _Param:
    def __init__(self, name, kind, ctype=None, nd=0, struct=None):
        self.name, self.kind, self.ctype, self.nd, self.struct = name, kind, ctype, nd, struct

    @property
    def nviews(self):
        return self.struct.count if self.struct else 1


class StencilInfo:
    """What the front end learned about one stencil function."""

    def __init__(self, name, ndims, index_names, gparams, scalars):
        self.name = name
        self.ndims = ndims
        self.index_names = index_names
        self.gparams = gparams      # [_Param] of the grid parameters
        self.grids = [(p.name, p.ctype if not p.struct else ps.PS_USER, p.nd) for p in gparams]
        self.scalars = scalars      # [(name, type)]
        self.base = []              # first view of each grid parameter
        self.view_type = []
        for p in gparams:
            self.base.append(len(self.view_type))
            if p.struct:
                for f in p.struct.fields:
                    self.view_type += [f.ctype] * f.count
            else:
                self.view_type.append(p.ctype)
        self.view_emits = [0] * len(self.view_type)
        self.view_reads_offset = [0] * len(self.view_type)
        self.axes = [None] * len(gparams)
        # What the staged (TMA plane ring) form needs: every read at
        # (x + a, y + b, z + c) with constants |a|, |b|, |c| <= 2, read offset
        # ranges per grid, and a single emit (see _staged_eligible).
        self.staged_ok = ndims == 3
        self.staged_reads = {}      # grid slot -> [lo[3], hi[3]]
        self.staged_rows = {}       # (slot, dy, dz) -> [dx min, dx max], in first-read order
        # Grid slots read with PSGridGetPeriodic: the staged form takes their
        # wrapped values from the pitched grid's refreshed halo (plain reads
        # of the same grid stay inside it or are checked, so they never see
        # the halo).
        self.staged_periodic = set()
        self.emit_count = 0
        self.emit_slot = None
        self.staged = False

    @property
    def grid_types(self):
        return [t for _, t, _ in self.grids]

    def _per_grid(self, per_view):
        return [int(any(per_view[self.base[i]:self.base[i] + p.nviews]))
                for i, p in enumerate(self.gparams)]

    @property
    def emits(self):
        """1 for each grid parameter that has an emitted view."""
        return self._per_grid(self.view_emits)

    @property
    def reads_offset(self):
        return self._per_grid(self.view_reads_offset)


def _params_of(fd, user):
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
        elif tn in user:
            nd, st = user[tn]
            out.append(_Param(p.name, "grid", None, nd, st))
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


def _member_chain(node):
    """(base, field name, [subscripts]) of `base.field[a][b]`, else None."""
    subs = []
    while isinstance(node, c_ast.ArrayRef):
        subs.append(node.subscript)
        node = node.name
    if isinstance(node, c_ast.StructRef) and node.type == "." and \
            isinstance(node.field, c_ast.ID):
        return node.name, node.field.name, subs[::-1]
    return None


def _field_var(gname, fname):
    return "%s__%s" % (gname, fname)


def _int(v):
    return c_ast.Constant("int", str(v))


class _Rewriter:
    """Rewrites the intrinsics of one function body in place."""

    def __init__(self, fname, params, info, functions):
        self.fname = fname
        self.index_names = [p.name for p in params if p.kind == "index"]
        gp = [p for p in params if p.kind == "grid"]
        self.grids = {p.name: (i, p) for i, p in enumerate(gp)}
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

    # -- views -----------------------------------------------------------
    def _mark(self, slot, lo, n, what):
        if self.info is None:
            return
        arr = self.info.view_emits if what == "emit" else self.info.view_reads_offset
        b = self.info.base[slot]
        for v in range(b + lo, b + lo + n):
            arr[v] = 1

    def _component(self, node, p, fname, subs):
        """(array variable, index expression, first component, components
        it may be) of member `fname[subs]` of a user-type grid."""
        f = p.struct.field(fname)
        if f is None:
            self.fail(node, "struct %s has no member %s" % (p.struct.name, fname))
        if len(subs) != len(f.dims):
            self.fail(node, "member %s of struct %s is read as an array: give all %d subscripts"
                      % (fname, p.struct.name, len(f.dims)))
        consts = [_const_int(e) for e in subs]
        if all(c is not None for c in consts):
            flat = 0
            for c, d in zip(consts, f.dims):
                if not 0 <= c < d:
                    self.fail(node, "subscript of %s out of its bounds" % fname)
                flat = flat * d + c
            return _field_var(p.name, fname), _int(flat), f.first + flat, 1
        expr = None
        for e, d in zip(subs, f.dims):
            expr = e if expr is None else c_ast.BinaryOp(
                "+", c_ast.BinaryOp("*", expr, _int(d)), e)
        return _field_var(p.name, fname), expr, f.first, f.count

    def _indices(self, node, p, idx):
        if len(idx) != p.nd:
            self.fail(node, "%s of a %d-D grid takes %d indices" % (node.name.name, p.nd, p.nd))
        # The reference's translator wants `index parameter +- constant`
        # (for its halo analysis, docs/programming.md:161-171); here any
        # integer expression is read (reads are bounds-checked), and a read
        # that is not at the point itself marks the view as read off the
        # point (no in-place update without red-black order).
        forms = [_index_form(e, self.index_names) for e in idx]
        at_point = len(idx) == len(self.index_names) and all(
            f is not None and f == (k, 0) for k, f in enumerate(forms))
        return forms, at_point

    def _record_axes(self, slot, forms):
        if self.info is not None and all(f is not None for f in forms) and \
                self.info.axes[slot] is None:
            self.info.axes[slot] = [f[0] for f in forms]

    def _point(self):
        return [c_ast.ID(n) for n in self.index_names] + [_int(0)] * (3 - len(self.index_names))

    def _staged_read(self, slot, p, forms, periodic):
        """Record a read for the staged form, or rule the form out."""
        if self.info is None:
            return
        if p.struct is not None or p.nd != 3 or len(forms) != 3 or \
                any(f is None or f[0] != k or abs(f[1]) > 2 for k, f in enumerate(forms)):
            self.info.staged_ok = False
            return
        if periodic:
            self.info.staged_periodic.add(slot)
        lo, hi = self.info.staged_reads.setdefault(slot, [[2, 2, 2], [-2, -2, -2]])
        for k, f in enumerate(forms):
            lo[k] = min(lo[k], f[1])
            hi[k] = max(hi[k], f[1])
        row = self.info.staged_rows.setdefault((slot, forms[1][1], forms[2][1]), [2, -2])
        row[0] = min(row[0], forms[0][1])
        row[1] = max(row[1], forms[0][1])

    def visit(self, node):
        ch = _member_chain(node)
        if ch is not None:
            base, fname, subs = ch
            if isinstance(base, c_ast.FuncCall) and isinstance(base.name, c_ast.ID) and \
                    base.name.name in ("PSGridGet", "PSGridGetPeriodic"):
                args = base.args.exprs if base.args else []
                slot, p = self.grid_arg(base, args[0] if args else None)
                if p.struct is not None:
                    return self.member_get(base, slot, p, args[1:], fname, subs)
            if isinstance(base, c_ast.ID) and base.name in self.grids:
                self.fail(node, "a member of a grid is only written by PSGridEmitUtype")
        if isinstance(node, c_ast.FuncCall) and isinstance(node.name, c_ast.ID) and \
                node.name.name == "PSGridEmitUtype":
            return self.emit_member(node)
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

    def member_get(self, call, slot, p, idx, fname, subs):
        idx = [self.visit(e) for e in idx]
        subs = [self.visit(e) for e in subs]
        forms, at_point = self._indices(call, p, idx)
        self._record_axes(slot, forms)
        var, sub, first, n = self._component(call, p, fname, subs)
        if self.info is not None:
            self.info.staged_ok = False
        if not at_point:
            self._mark(slot, first, n, "read")
        helper = "__psb_getp" if call.name.name == "PSGridGetPeriodic" else "__psb_get"
        if n == 1:
            return c_ast.FuncCall(c_ast.ID(helper), c_ast.ExprList(
                [c_ast.ArrayRef(c_ast.ID(var), sub)] + idx), call.coord)
        # A subscript computed at run time is checked against the member.
        return c_ast.FuncCall(c_ast.ID(helper + "_c"), c_ast.ExprList(
            [c_ast.ID(var), _int(n), sub] + idx), call.coord)

    def emit_member(self, node):
        args = node.args.exprs if node.args else []
        if len(args) != 2:
            self.fail(node, "PSGridEmitUtype takes a grid member and a value")
        ch = _member_chain(args[0])
        if ch is None or not isinstance(ch[0], c_ast.ID) or ch[0].name not in self.grids or \
                self.grids[ch[0].name][1].struct is None:
            self.fail(node, "the first argument of PSGridEmitUtype must be a member of a grid "
                            "of a user-defined point type")
        slot, p = self.grids[ch[0].name]
        if p.nd != len(self.index_names):
            self.fail(node, "PSGridEmitUtype into a %d-D grid from a %d-D stencil" %
                      (p.nd, len(self.index_names)))
        subs = [self.visit(e) for e in ch[2]]
        value = self.visit(args[1])
        var, sub, first, n = self._component(node, p, ch[1], subs)
        if self.info is not None:
            self.info.staged_ok = False
        self._mark(slot, first, n, "emit")
        if n == 1:
            return c_ast.FuncCall(c_ast.ID("__psb_emit"), c_ast.ExprList(
                [c_ast.ArrayRef(c_ast.ID(var), sub)] + self._point() + [value]), node.coord)
        return c_ast.FuncCall(c_ast.ID("__psb_emit_c"), c_ast.ExprList(
            [c_ast.ID(var), _int(n), sub] + self._point() + [value]), node.coord)

    def _field_args(self, p):
        return [c_ast.ID(_field_var(p.name, f.name)) for f in p.struct.fields]

    def call(self, node):
        fn = node.name.name
        args = node.args.exprs if node.args else []
        if fn in ("PSGridGet", "PSGridGetPeriodic"):
            slot, p = self.grid_arg(node, args[0] if args else None)
            idx = args[1:]
            forms, at_point = self._indices(node, p, idx)
            self._record_axes(slot, forms)
            if not at_point:
                self._mark(slot, 0, p.nviews, "read")
            per = fn == "PSGridGetPeriodic"
            self._staged_read(slot, p, forms, per)
            if p.struct is not None:   # the whole record
                helper = "__psb_load%s_%s" % ("p" if per else "", p.struct.name)
                return c_ast.FuncCall(c_ast.ID(helper), c_ast.ExprList(
                    self._field_args(p) + idx), node.coord)
            helper = "__psb_getp" if per else "__psb_get"
            return c_ast.FuncCall(c_ast.ID(helper), c_ast.ExprList([c_ast.ID(p.name)] + idx),
                                  node.coord)
        if fn == "PSGridEmit":
            if len(args) != 2:
                self.fail(node, "PSGridEmit takes a grid and a value")
            slot, p = self.grid_arg(node, args[0])
            if p.nd != len(self.index_names):
                self.fail(node, "PSGridEmit into a %d-D grid from a %d-D stencil" %
                          (p.nd, len(self.index_names)))
            self._mark(slot, 0, p.nviews, "emit")
            if self.info is not None:
                self.info.emit_count += 1
                self.info.emit_slot = slot
                if p.struct is not None:
                    self.info.staged_ok = False
            if p.struct is not None:
                return c_ast.FuncCall(c_ast.ID("__psb_store_" + p.struct.name), c_ast.ExprList(
                    self._field_args(p) + self._point() + [args[1]]), node.coord)
            return c_ast.FuncCall(c_ast.ID("__psb_emit"), c_ast.ExprList(
                [c_ast.ID(p.name)] + self._point() + [args[1]]), node.coord)
        if fn == "PSGridDim":
            if len(args) != 2:
                self.fail(node, "PSGridDim takes a grid and a dimension")
            slot, p = self.grid_arg(node, args[0])
            g = c_ast.ID(p.name) if p.struct is None else c_ast.ArrayRef(
                c_ast.ID(_field_var(p.name, p.struct.fields[0].name)), _int(0))
            return c_ast.FuncCall(c_ast.ID("__psb_dim"), c_ast.ExprList([g, args[1]]), node.coord)
        if fn.startswith("PS"):
            self.fail(node, "%s is not available inside a stencil function" % fn)
        if fn in self.functions:
            # A grid of a point type is passed on as its field arrays.
            out = []
            for a in args:
                if isinstance(a, c_ast.ID) and a.name in self.grids and \
                        self.grids[a.name][1].struct is not None:
                    out += self._field_args(self.grids[a.name][1])
                else:
                    out.append(a)
            if node.args:
                node.args.exprs = out
            return node
        if fn in _MATH_DOUBLE:
            dargs = [c_ast.Cast(c_ast.Typename(None, [], None, c_ast.TypeDecl(
                None, [], None, c_ast.IdentifierType(["double"]))), a) for a in args]
            return c_ast.FuncCall(c_ast.ID(fn), c_ast.ExprList(dargs), node.coord)
        return node


_HELPERS = r"""
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include "physis_b200.h"
#include "k_generic_tma.cuh"

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

// Stores at the current point (unused index parameters are 0).
template <typename T, typename V>
__device__ __forceinline__ void __psb_emit(const __psb_grid<T> &g, int i, int j, int k, V v) {
  g.p[i + j * g.sy + k * g.sz] = (T)v;
}

// Members of point types indexed at run time: a subscript outside the member
// reads 0 / stores nothing and sets PSB_ERR_BOUNDS.
template <typename T>
__device__ __forceinline__ T __psb_get_c(const __psb_grid<T> *f, int n, int c, int i, int j = 0,
                                         int k = 0) {
  if ((unsigned)c >= (unsigned)n) {
    atomicExch(f[0].err, (int)PSB_ERR_BOUNDS);
    return T(0);
  }
  return __psb_get(f[c], i, j, k);
}
template <typename T>
__device__ __forceinline__ T __psb_getp_c(const __psb_grid<T> *f, int n, int c, int i, int j = 0,
                                          int k = 0) {
  if ((unsigned)c >= (unsigned)n) {
    atomicExch(f[0].err, (int)PSB_ERR_BOUNDS);
    return T(0);
  }
  return __psb_getp(f[c], i, j, k);
}
template <typename T, typename V>
__device__ __forceinline__ void __psb_emit_c(const __psb_grid<T> *f, int n, int c, int i, int j,
                                             int k, V v) {
  if ((unsigned)c >= (unsigned)n) {
    atomicExch(f[0].err, (int)PSB_ERR_BOUNDS);
    return;
  }
  __psb_emit(f[c], i, j, k, v);
}

template <typename T>
__device__ __forceinline__ int __psb_dim(const __psb_grid<T> &g, int d) {
  return d == 0 ? g.n0 : (d == 1 ? g.n1 : g.n2);
}

// Staged form (a stencil function run over the library's TMA plane ring):
// a grid read from the staged window at an offset from the point in row r,
// column v of the thread's block, and the grid emitted into, whose value
// goes to that point's result.
// A read grid of the staged form: the rows the function reads around the
// current row of the thread's block, in registers (L::id maps a row's grid,
// dy and dz to its index), and the point's column v in that row. Unchecked
// (C false): the library runs it only when every read the function can make
// over the map's domain lies inside its grid. Checked (C true): a read that
// leaves the point on an axis is tested against the grid there and, outside,
// reads 0 and marks the thread's flag (*bad), which the program turns into
// PSB_ERR_BOUNDS once per thread like the function's own form reports it.
// The library runs it only with the domain inside the grid, so a read at
// the point's own coordinate on an axis needs no test (the offsets are
// constants after inlining, so each read keeps the tests of its own axes).
// The test is a select, not a branch, so the points of a thread's block
// still schedule together.
template <typename T, class L, bool C>
struct __psb_rgrid {
  const psb::GtRow<T> *rows;
  int slot, v, x, y, z;
  int n0, n1, n2;
  int *bad;
};

template <typename T, class L, bool C>
__device__ __forceinline__ T __psb_get(const __psb_rgrid<T, L, C> &g, int i, int j = 0,
                                       int k = 0) {
  const int dx = i - g.x, dy = j - g.y, dz = k - g.z;
  const T val = g.rows[L::id(g.slot, dy, dz)].e[2 + dx + g.v];
  if (!C) return val;
  const bool out = ((dx != 0) & ((unsigned)i >= (unsigned)g.n0)) |
                   ((dy != 0) & ((unsigned)j >= (unsigned)g.n1)) |
                   ((dz != 0) & ((unsigned)k >= (unsigned)g.n2));
  *g.bad |= (int)out;
  return out ? T(0) : val;
}

// A periodic read: the window holds the wrapped values (the library
// refreshes the pitched grid's halo first), so it needs no check.
template <typename T, class L, bool C>
__device__ __forceinline__ T __psb_getp(const __psb_rgrid<T, L, C> &g, int i, int j = 0,
                                        int k = 0) {
  return g.rows[L::id(g.slot, j - g.y, k - g.z)].e[2 + (i - g.x) + g.v];
}

template <typename T, class L, bool C>
__device__ __forceinline__ int __psb_dim(const __psb_rgrid<T, L, C> &g, int d) {
  return d == 0 ? g.n0 : (d == 1 ? g.n1 : g.n2);
}

template <typename T>
struct __psb_ogrid {
  T *out;
  int n0, n1, n2;
};

template <typename T, typename V>
__device__ __forceinline__ void __psb_emit(const __psb_ogrid<T> &g, int, int, int, V v) {
  *g.out = (T)v;
}

template <typename T>
__device__ __forceinline__ int __psb_dim(const __psb_ogrid<T> &g, int d) {
  return d == 0 ? g.n0 : (d == 1 ? g.n1 : g.n2);
}
"""


def _struct_helpers(st):
    """Whole-record load (plain and periodic) and store of a point type."""
    params = ", ".join("const __psb_grid<%s> *f_%s" % (_CTYPE[f.ctype], f.name)
                       for f in st.fields)
    out = []
    for per in (False, True):
        body = []
        for f in st.fields:
            for flat in range(f.count):
                sub, r = "", flat
                for d in reversed(f.dims):
                    sub = "[%d]" % (r % d) + sub
                    r //= d
                body.append("  v.%s%s = %s(f_%s[%d], i, j, k);" % (
                    f.name, sub, "__psb_getp" if per else "__psb_get", f.name, flat))
        out.append("__device__ __forceinline__ struct %s __psb_load%s_%s(%s, int i, int j = 0, "
                   "int k = 0) {\n  struct %s v;\n%s\n  return v;\n}" % (
                       st.name, "p" if per else "", st.name, params, st.name, "\n".join(body)))
    body = []
    for f in st.fields:
        for flat in range(f.count):
            sub, r = "", flat
            for d in reversed(f.dims):
                sub = "[%d]" % (r % d) + sub
                r //= d
            body.append("  __psb_emit(f_%s[%d], i, j, k, v.%s%s);" % (f.name, flat, f.name, sub))
    out.append("__device__ __forceinline__ void __psb_store_%s(%s, int i, int j, int k, "
               "const struct %s &v) {\n%s\n}" % (st.name, params, st.name, "\n".join(body)))
    return "\n\n".join(out)


def _signature(fname, params):
    out = []
    for p in params:
        if p.kind == "index":
            out.append("const int %s" % p.name)
        elif p.kind == "grid" and p.struct is not None:
            for f in p.struct.fields:
                out.append("const __psb_grid<%s> *%s" % (_CTYPE[f.ctype],
                                                          _field_var(p.name, f.name)))
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


def _reachable(funcs, user):
    """The stencil functions and the functions they call (directly or not),
    in source order; the rest of the program (main, I/O) is host code."""
    by_name = {f.decl.name: f for f in funcs}
    todo = [f.decl.name for f in funcs if _is_stencil(_params_of(f, user))]
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
    text, user_decl = _preprocess(source)
    try:
        ast = c_parser.CParser().parse(_prelude() + text, filename="<dsl>")
    except Exception as e:  # pycparser raises ParseError with a location
        raise DSLError("cannot parse the stencil source: %s" % e) from None
    gen = c_generator.CGenerator()
    structs = _struct_defs(ast)
    user = {}
    for tname, (nd, sname) in user_decl.items():
        if sname not in structs:
            raise DSLError("%s: struct %s is not defined with float/double/int/long members "
                           "of fixed size" % (tname, sname))
        user[tname] = (nd, structs[sname])
    funcs = [n for n in ast.ext if isinstance(n, c_ast.FuncDef)]
    names = {f.decl.name for f in funcs}
    funcs = _reachable(funcs, user)
    infos = {}
    parts = [_HELPERS]
    # Point types and their record helpers, then declarations first, so
    # functions may call each other in any order.
    used = []
    for nd, st in user.values():
        if st not in used:
            used.append(st)
    for n in ast.ext:
        if isinstance(n, c_ast.Decl) and isinstance(getattr(n, "type", None), c_ast.Struct) \
                and n.type.decls:
            parts.append(gen.visit(n) + ";")
    for st in used:
        parts.append(_struct_helpers(st))
    decls = []
    bodies = []
    for fd in funcs:
        fname = fd.decl.name
        if fname == "main":
            continue
        params = _params_of(fd, user)
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
            gparams = [p for p in params if p.kind == "grid"]
            scalars = [(p.name, p.ctype) for p in params if p.kind == "scalar"]
            info = StencilInfo(fname, nidx, [p.name for p in params[:nidx]], gparams, scalars)
            if len(gparams) > ps.PSB_MAX_GRIDS or len(scalars) > ps.PSB_MAX_PARAMS or \
                    len(info.view_type) > ps.PSB_MAX_VIEWS:
                raise DSLError("%s: too many grid, component or scalar parameters" % fname)
            _Rewriter(fname, params, info, names).visit(fd.body)
            for slot, p in enumerate(gparams):
                if info.axes[slot] is None:
                    info.axes[slot] = list(range(p.nd))
            info.staged = _staged_eligible(info, fd.body)
            infos[fname] = info
            sig = _signature(fname, params)
        else:
            if any(p.kind == "grid" for p in params):
                raise DSLError("%s: a function that takes grids is a stencil function and "
                               "begins with its `const int` index parameters" % fname)
            _Rewriter(fname, params, None, names).visit(fd.body)
            sig = "__device__ " + gen.visit(fd.decl).rstrip(";")
        decls.append(sig + ";")
        body = gen.visit(fd.body)
        bodies.append(sig + "\n" + body)
        if fname in infos and infos[fname].staged:
            bodies.append(_staged_function(infos[fname], params, body))
    if not infos:
        raise DSLError("no stencil function (`void f(const int x, ..., grids, ...)`) found")
    parts.append("\n".join(decls))
    parts.append("\n\n".join(bodies))
    for info in infos.values():
        if info.staged:
            parts.append(_staged_entry(info))
        parts.append(_entry(info))
    return "\n\n".join(parts) + "\n", infos


def _staged_eligible(info, body):
    """Whether the function has a staged form: 3-D, one element type (float
    or double) over primitive 3-D grids, every read at constant offsets
    within +-2 of the point, one emit, as a statement of the body's top
    level with no return before it, into a grid it does not read."""
    if not info.staged_ok or info.emit_count != 1 or info.emit_slot is None:
        return False
    if any(p.struct is not None or p.nd != 3 for p in info.gparams):
        return False
    types = {p.ctype for p in info.gparams}
    if len(types) != 1 or types.pop() not in (ps.PS_FLOAT, ps.PS_DOUBLE):
        return False
    if not info.staged_reads or info.emit_slot in info.staged_reads or len(info.scalars) > 32:
        return False
    items = body.block_items or []
    at = [i for i, it in enumerate(items) if isinstance(it, c_ast.FuncCall) and
          isinstance(it.name, c_ast.ID) and it.name.name == "__psb_emit"]
    if len(at) != 1:
        return False

    class _Returns(c_ast.NodeVisitor):
        found = False

        def visit_Return(self, node):
            self.found = True

    r = _Returns()
    for it in items[:at[0]]:
        r.visit(it)
    return not r.found


def _staged_function(info, params, body):
    """The function again, its grids as template parameters: staged handles
    (reads from the plane ring, the emit into the point's result)."""
    tpl, args, g = [], [], 0
    for p in params:
        if p.kind == "index":
            args.append("const int %s" % p.name)
        elif p.kind == "grid":
            tpl.append("class __G%d" % g)
            args.append("const __G%d &%s" % (g, p.name))
            g += 1
        elif p.kind == "scalar":
            args.append("%s %s" % (_CTYPE[p.ctype], p.name))
    return "template <%s>\n__device__ __forceinline__ void %s__staged(%s)\n%s" % (
        ", ".join(tpl), info.name, ", ".join(args), body)


def _staged_entry(info):
    """The point-wise program, kernels and launchers of the staged form,
    unchecked and checked (psb_dsl_staged_<name>, psb_dsl_staged_checked_<name>).

    For each row of the thread's block the rows the function reads -- one
    per (grid, dy, dz) -- are loaded into registers as the generic packed
    form does (a 16-byte load per thread, x neighbours from the adjacent
    lanes); every read of the function then resolves, at compile time, to a
    register of one of those rows. The checked form tests the reads that
    leave the point against their grids first (rows outside a grid hold
    whatever the window holds there and are never returned)."""
    n = info.name
    t = _CTYPE[info.gparams[0].ctype]
    rows = list(info.staged_rows.items())
    ids = " : ".join("(slot == %d && dy == %d && dz == %d) ? %d" % (sl, dy, dz, k)
                     for k, ((sl, dy, dz), _) in enumerate(rows)) + " : 0"
    loads = []
    for k, ((sl, dy, dz), (dxlo, dxhi)) in enumerate(rows):
        loads.append(
            "{ int sl = at.slot0 + %d - at.zmin; if (sl >= at.S) sl -= at.S;\n"
            "          psb::gt_row_load(reinterpret_cast<const T *>(at.ring + (size_t)sl * at.sbytes) + "
            "tab.slot_grid[%d] * at.plane_elems + at.thr_off + (r + %d) * at.bx, lane, %s, %s, "
            "rows[%d]); }" % (dz, sl, dy, "true" if dxhi > 0 else "false",
                              "true" if dxlo < 0 else "false", k))
    handles, args = [], []
    for slot in range(len(info.gparams)):
        dims = ", ".join("tab.slot_dims[%d][%d]" % (slot, k) for k in range(3))
        if slot == info.emit_slot:
            handles.append("const __psb_ogrid<T> g%d{&acc.v[r][v], %s};" % (slot, dims))
        else:
            handles.append("const __psb_rgrid<T, __psb_rows_%s, C> g%d{rows, %d, v, x, y, at.z, "
                           "%s, &bad};" % (n, slot, slot, dims))
        args.append("g%d" % slot)
    for k, (_, st) in enumerate(info.scalars):
        args.append("(%s)tab.coef[%d]" % (_CTYPE[st], k))
    return """
struct __psb_rows_{n} {{
  static __device__ __forceinline__ constexpr int id(int slot, int dy, int dz) {{
    return {ids};
  }}
}};

template <bool C>
struct __psb_prog_{n} {{
  static constexpr bool kCompiled = true;
  static constexpr bool kPoints = true;
  template <typename T>
  static __device__ __forceinline__ void eval(const psb::GtTable &, const unsigned char *, int,
                                              int, int, int, int, int, psb::GtBlk<T> &) {{}}
  template <typename T>
  static __device__ __forceinline__ void eval_points(const psb::GtTable &tab,
                                                     const psb::GtAt &at, psb::GtBlk<T> &acc) {{
    const int lane = threadIdx.x & 31;
    int bad = 0;  // a checked read of this thread's block left its grid
#pragma unroll
    for (int r = 0; r < psb::kGtVY; r++) {{
      psb::GtRow<T> rows[{nrows}];  // every lane loads: the rows share values by shuffles
      {loads}
      const int y = at.y + r;
      if (y < at.lo1 || y >= at.hi1) continue;
#pragma unroll
      for (int v = 0; v < 16 / (int)sizeof(T); v++) {{
        const int x = at.x + v;
        if (x < at.lo0 || x >= at.hi0) continue;
        {handles}
        {n}__staged(x, y, at.z, {args});
      }}
    }}
    if (C && bad) atomicExch(tab.read_err, (int)PSB_ERR_BOUNDS);
  }}
}};

extern "C" __global__ void __launch_bounds__(psb::kGtThreads, 2) __psb_staged_kernel_{n}(
    const __grid_constant__ psb::GtMaps maps, const __grid_constant__ psb::GtTable tab,
    psb::GridView out, psb::Dom3 d, const __grid_constant__ psb::GtGeom geo, int *err) {{
  psb::gt_body<{t}, __psb_prog_{n}<false>>(maps, tab, out, d, geo, err);
}}

extern "C" __global__ void __launch_bounds__(psb::kGtThreads, 2) __psb_staged_checked_kernel_{n}(
    const __grid_constant__ psb::GtMaps maps, const __grid_constant__ psb::GtTable tab,
    psb::GridView out, psb::Dom3 d, const __grid_constant__ psb::GtGeom geo, int *err) {{
  psb::gt_body<{t}, __psb_prog_{n}<true>>(maps, tab, out, d, geo, err);
}}

typedef void (*__psb_staged_kernel_t_{n})(psb::GtMaps, psb::GtTable, psb::GridView, psb::Dom3,
                                          psb::GtGeom, int *);

static psb_status __psb_staged_launch_{n}(__psb_staged_kernel_t_{n} k, unsigned *configured,
                                          const void *maps, const void *table, const void *out,
                                          const void *dom, const void *geo, int *err,
                                          unsigned blocks, unsigned smem, void *stream) {{
  if (smem > *configured) {{
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess)
      return PSB_ERR_CUDA;
    *configured = smem;
  }}
  k<<<blocks, psb::kGtThreads, smem, (cudaStream_t)stream>>>(
      *(const psb::GtMaps *)maps, *(const psb::GtTable *)table, *(const psb::GridView *)out,
      *(const psb::Dom3 *)dom, *(const psb::GtGeom *)geo, err);
  return cudaGetLastError() == cudaSuccess ? PSB_OK : PSB_ERR_CUDA;
}}

extern "C" psb_status psb_dsl_staged_{n}(const void *maps, const void *table, const void *out,
                                         const void *dom, const void *geo, int *err,
                                         unsigned blocks, unsigned smem, void *stream) {{
  static unsigned configured = 0;
  return __psb_staged_launch_{n}(__psb_staged_kernel_{n}, &configured, maps, table, out, dom,
                                 geo, err, blocks, smem, stream);
}}

extern "C" psb_status psb_dsl_staged_checked_{n}(const void *maps, const void *table,
                                                 const void *out, const void *dom,
                                                 const void *geo, int *err, unsigned blocks,
                                                 unsigned smem, void *stream) {{
  static unsigned configured = 0;
  return __psb_staged_launch_{n}(__psb_staged_checked_kernel_{n}, &configured, maps, table, out,
                                 dom, geo, err, blocks, smem, stream);
}}
""".format(n=n, t=t, ids=ids, nrows=len(rows), loads="\n      ".join(loads),
           handles="\n        ".join(handles), args=", ".join(args))


def _read_ranges(info):
    """Flat lo and hi read offsets per grid parameter for the descriptor
    (lo 1 > hi 0 on every axis: not read by the staged form)."""
    lo, hi = [], []
    for slot in range(len(info.gparams)):
        r = info.staged_reads.get(slot) if info.staged else None
        lo += r[0] if r else [1, 1, 1]
        hi += r[1] if r else [0, 0, 0]
    return lo, hi


def _entry(info):
    """The kernel, launch and describe functions of one stencil function."""
    n = info.name
    binds = []
    args = ["x", "y", "z"][:info.ndims]
    for slot, p in enumerate(info.gparams):
        b = info.base[slot]
        if p.struct is None:
            t = _CTYPE[p.ctype]
            binds.append("  const __psb_grid<%s> g%d = __psb_bind<%s>(A.views[%d], A.error);" %
                         (t, slot, t, b))
            args.append("g%d" % slot)
            continue
        for f in p.struct.fields:
            t = _CTYPE[f.ctype]
            items = ", ".join("__psb_bind<%s>(A.views[%d], A.error)" % (t, b + f.first + k)
                              for k in range(f.count))
            binds.append("  const __psb_grid<%s> g%d__%s[%d] = {%s};" % (t, slot, f.name, f.count,
                                                                          items))
            args.append("g%d__%s" % (slot, f.name))
    for k, (sname, t) in enumerate(info.scalars):
        args.append("(%s)A.params[%d]" % (_CTYPE[t], k))

    def arr(vals):
        return ", ".join(str(v) for v in vals) or "0"

    comps = [p.nviews for p in info.gparams]
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
  const int gt[] = {{{gt}}}, gn[] = {{{gn}}}, gc[] = {{{gc}}};
  const int vt[] = {{{vt}}}, ve[] = {{{ve}}}, vr[] = {{{vr}}}, pt[] = {{{pt}}};
  d->ndims = {nd};
  d->ngrids = {ng};
  for (int i = 0; i < {ng}; i++) {{
    d->grid_type[i] = gt[i];
    d->grid_ndims[i] = gn[i];
    d->grid_components[i] = gc[i];
  }}
  d->nviews = {nv};
  for (int v = 0; v < {nv}; v++) {{
    d->view_type[v] = vt[v];
    d->view_emits[v] = ve[v];
    d->view_reads_offset[v] = vr[v];
  }}
  d->nparams = {np};
  for (int i = 0; i < {np}; i++) d->param_type[i] = pt[i];
  d->launch = psb_dsl_launch_{n};
  const int rlo[] = {{{rlo}}}, rhi[] = {{{rhi}}};
  for (int i = 0; i < PSB_MAX_GRIDS; i++)
    for (int k = 0; k < 3; k++) {{
      d->read_lo[i][k] = i < {ng} ? rlo[3 * i + k] : 1;
      d->read_hi[i][k] = i < {ng} ? rhi[3 * i + k] : 0;
    }}
  d->staged_type = {stype};
  d->staged_emit = {semit};
  d->staged = {sfn};
  d->staged_checked = {cfn};
  const int rper[] = {{{rper}}};
  for (int i = 0; i < PSB_MAX_GRIDS; i++) d->read_periodic[i] = i < {ng} ? rper[i] : 0;
}}
""".format(rlo=arr(_read_ranges(info)[0]), rhi=arr(_read_ranges(info)[1]),
           stype=info.gparams[0].ctype if info.staged else 0,
           semit=info.emit_slot if info.staged else 0,
           sfn=("psb_dsl_staged_%s" % n) if info.staged else "nullptr",
           cfn=("psb_dsl_staged_checked_%s" % n) if info.staged else "nullptr",
           rper=arr(1 if info.staged and slot in info.staged_periodic else 0
                    for slot in range(len(info.grids))),
           n=n, binds="\n".join(binds), args=", ".join(args), gt=arr(info.grid_types),
           gn=arr(nd for _, _, nd in info.grids), gc=arr(comps), vt=arr(info.view_type),
           ve=arr(info.view_emits), vr=arr(info.view_reads_offset),
           pt=arr(t for _, t in info.scalars), nd=info.ndims, ng=len(info.grids),
           nv=len(info.view_type), np=len(info.scalars))


_NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
               "-fmad=false", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared"]
CSRC = os.path.join(HERE, "csrc")
# Device headers the staged form compiles against (part of the cache key).
_STAGED_HEADERS = ["k_generic_tma.cuh", "device.cuh", "views.h", "internal.h"]


def build_library(cuda_source, cache_dir=None):
    """Compile generated source for sm_100a into a shared library; returns
    its path. Libraries are cached by a hash of the source, the ABI header
    they are compiled against (the launch arguments' layout) and the flags."""
    cache_dir = cache_dir or DEFAULT_CACHE
    os.makedirs(cache_dir, exist_ok=True)
    h = hashlib.sha256(cuda_source.encode())
    with open(os.path.join(INCLUDE, "physis_b200.h"), "rb") as f:
        h.update(f.read())
    for name in _STAGED_HEADERS:
        with open(os.path.join(CSRC, name), "rb") as f:
            h.update(f.read())
    h.update(" ".join(_NVCC_FLAGS).encode())
    key = h.hexdigest()[:20]
    so = os.path.join(cache_dir, "libpsb_dsl_%s.so" % key)
    if os.path.exists(so):
        return so
    # Unique names per build: the same source may be built by several
    # threads or processes at once; the finished library is renamed in place.
    tag = "%d.%d" % (os.getpid(), threading.get_ident())
    cu = os.path.join(cache_dir, "psb_dsl_%s.%s.cu" % (key, tag))
    with open(cu, "w") as f:
        f.write(cuda_source)
    tmp = so + ".tmp" + tag
    cmd = [NVCC] + _NVCC_FLAGS + ["-I" + INCLUDE, "-I" + CSRC, cu, "-o", tmp]
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
