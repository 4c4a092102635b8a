"""The system-test stencils as DSL stencil functions for the front end.

Each entry is a stencil function in the reference's C DSL (written for these
tests, not taken from the reference) that computes what the matching case of
cases.py computes -- the same reads, in the same order, in the same types --
so the compiled kernel must print exactly the reference's known-answer
output. Entries: name -> (DSL source, name of the stencil function, scalars
passed to PSStencilMap).
"""
from tests.golden import cases as C

# Offsets of the reads, in the order each reference test sums them.
_O7 = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, -1), (0, 0, 1)]
_O7P = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]


def _at(var, d):
    return var if d == 0 else "%s %s %d" % (var, "+" if d > 0 else "-", abs(d))


def _read(grid, off, periodic=False, axes="xyz"):
    fn = "PSGridGetPeriodic" if periodic else "PSGridGet"
    return "%s(%s, %s)" % (fn, grid, ", ".join(_at(a, d) for a, d in zip(axes, off)))


def _sum_stencil(name, gtype, ctype, offs, periodic=False, nd=3):
    axes = "xyz"[:nd]
    idx = ", ".join("const int %s" % a for a in axes)
    reads = "\n      + ".join(_read("in", o[:nd], periodic, axes) for o in offs)
    return """
void %s(%s, PSGrid%dD%s in, PSGrid%dD%s out) {
  %s acc = %s;
  PSGridEmit(out, acc);
}
""" % (name, idx, nd, gtype, nd, gtype, ctype, reads)


def _inplace_stencil(name, offs, periodic):
    reads = "\n      + ".join(_read("u", o, periodic) for o in offs)
    return """
void %s(const int x, const int y, const int z, PSGrid3DFloat u) {
  float acc = %s;
  PSGridEmit(u, acc);
}
""" % (name, reads)


_NEUMANN = """
/* Zero-flux faces: a neighbour outside the grid is replaced by the point. */
static void neumann7(const int x, const int y, const int z,
                     PSGrid3DFloat src, PSGrid3DFloat dst,
                     float ce, float cw, float cn, float cs,
                     float ct, float cb, float cc) {
  const int lx = PSGridDim(src, 0) - 1, ly = PSGridDim(src, 1) - 1, lz = PSGridDim(src, 2) - 1;
  float here = PSGridGet(src, x, y, z);
  float west = x > 0 ? PSGridGet(src, x - 1, y, z) : here;
  float east = x < lx ? PSGridGet(src, x + 1, y, z) : here;
  float north, south, below, above;
  if (y > 0) north = PSGridGet(src, x, y - 1, z); else north = here;
  if (y < ly) south = PSGridGet(src, x, y + 1, z); else south = here;
  if (z > 0) below = PSGridGet(src, x, y, z - 1); else below = here;
  if (z < lz) above = PSGridGet(src, x, y, z + 1); else above = here;
  PSGridEmit(dst, cc * here + cw * west + ce * east + cs * south + cn * north
                  + cb * below + ct * above);
}
"""

_TYPE_MIX = """
void mixed_types(const int x, const int y, const int z, PSGrid3DFloat f,
                 PSGrid3DDouble d, PSGrid3DInt w) {
  double s = (double)PSGridGet(f, x, y, z);
  s = s + (double)PSGridGet(f, x + 1, y, z);
  s = s + (double)PSGridGet(f, x - 1, y, z);
  s = s + (double)PSGridGet(f, x, y + 1, z);
  s = s + (double)PSGridGet(f, x, y - 1, z);
  s = s + (double)PSGridGet(f, x, y, z - 1);
  s = s + (double)PSGridGet(f, x, y, z + 1);
  PSGridEmit(d, s * PSGridGet(w, x, y, z));
}
"""

_CLAMPED = """
static int clamp_index(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

void clamped7(const int x, const int y, const int z, PSGrid3DFloat a, PSGrid3DFloat b) {
  int nx = PSGridDim(a, 0), ny = PSGridDim(a, 1), nz = PSGridDim(a, 2);
  float v = PSGridGet(a, x, y, z)
      + PSGridGet(a, clamp_index(x - 1, nx), y, z)
      + PSGridGet(a, clamp_index(x + 1, nx), y, z)
      + PSGridGet(a, x, clamp_index(y + 1, ny), z)
      + PSGridGet(a, x, clamp_index(y - 1, ny), z)
      + PSGridGet(a, x, y, clamp_index(z - 1, nz))
      + PSGridGet(a, x, y, clamp_index(z + 1, nz));
  PSGridEmit(b, v);
}
"""

_MIXED1 = """
void weighted_x(const int x, const int y, const int z,
                PSGrid3DFloat u, PSGrid3DFloat v, PSGrid1DFloat k) {
  float t0 = PSGridGet(u, x, y, z) * PSGridGet(k, x);
  float t1 = PSGridGet(u, x - 1, y, z) * PSGridGet(k, x - 1);
  float t2 = PSGridGet(u, x + 1, y, z) * PSGridGet(k, x + 1);
  PSGridEmit(v, t0 + t1 + t2);
}
"""

_MIXED2 = """
void weighted_xyz(const int x, const int y, const int z, PSGrid3DFloat u,
                  PSGrid3DFloat v, PSGrid1DFloat kx, PSGrid1DFloat ky, PSGrid1DFloat kz) {
  float r = PSGridGet(u, x, y, z)
      + PSGridGet(u, x - 1, y, z) * PSGridGet(kx, x - 1)
      + PSGridGet(u, x + 1, y, z) * PSGridGet(kx, x + 1)
      + PSGridGet(u, x, y - 1, z) * PSGridGet(ky, y - 1)
      + PSGridGet(u, x, y + 1, z) * PSGridGet(ky, y + 1)
      + PSGridGet(u, x, y, z - 1) * PSGridGet(kz, z - 1)
      + PSGridGet(u, x, y, z + 1) * PSGridGet(kz, z + 1);
  PSGridEmit(v, r);
}
"""

_MIXED3 = """
void weighted_planes(const int x, const int y, const int z, PSGrid3DFloat u,
                     PSGrid3DFloat v, PSGrid1DFloat kx, PSGrid2DFloat kyz) {
  float r = PSGridGet(u, x, y, z)
      + PSGridGet(u, x - 1, y, z) * PSGridGet(kx, x - 1)
      + PSGridGet(u, x + 1, y, z) * PSGridGet(kx, x + 1)
      + PSGridGet(u, x, y - 1, z) * PSGridGet(kyz, y - 1, z)
      + PSGridGet(u, x, y + 1, z) * PSGridGet(kyz, y + 1, z)
      + PSGridGet(u, x, y, z - 1) * PSGridGet(kyz, y, z - 1)
      + PSGridGet(u, x, y, z + 1) * PSGridGet(kyz, y, z + 1);
  PSGridEmit(v, r);
}
"""

_ASYM_P = """
void lopsided(const int x, const int y, const int z, PSGrid3DFloat p, PSGrid3DFloat q) {
  float s = PSGridGet(p, x, y, z) + PSGridGet(p, x - 1, y, z);
  s = s + PSGridGetPeriodic(p, x + 2, y, z);
  PSGridEmit(q, s);
}
"""


_BRANCHES = """
/* Reads under data-independent conditions (x at the faces, x parity). */
void branches(const int x, const int y, const int z, PSGrid3DFloat in, PSGrid3DFloat out) {
  const float mid = PSGridGet(in, x, y, z);
  float acc = 0.0f;
  if (x > 0) acc = PSGridGet(in, x - 1, y, z);
  acc += x > 0 ? PSGridGet(in, x - 1, y, z) : PSGridGet(in, x, y, z);
  acc += x > 0 ? PSGridGet(in, x - 1, y, z) : mid;
  if (x > 0 && x < PSGridDim(in, 0) - 1)
    acc += PSGridGet(in, x - 1, y, z) + PSGridGet(in, x + 1, y, z);
  else
    acc += PSGridGet(in, x, y, z);
  if ((x & 1) == 0) acc += PSGridGet(in, x, y, z);
  PSGridEmit(out, mid + acc);
}
"""


# Point-type cases: (DSL source, [(function, grid slots)] applied in order each
# iteration, iterations, numpy record dtype, initial values per component as
# `i + offset` (None: 0), grids, dumped grid, dumped components (field, flat
# index)). The domain is the interior [1, N-1) in every case.
_VEC3 = """
struct Vec3 { float a; float b; float c; };
DeclareGrid3D(Vec3, struct Vec3);

void smooth3(const int x, const int y, const int z, PSGrid3DVec3 src, PSGrid3DVec3 dst) {
  float sa = (PSGridGet(src, x, y, z).a + PSGridGet(src, x + 1, y, z).a
              + PSGridGet(src, x - 1, y, z).a) / 3.3f;
  float sb = (PSGridGet(src, x, y, z).b + PSGridGet(src, x, y + 1, z).b
              + PSGridGet(src, x, y - 1, z).b + PSGridGet(src, x, y, z + 1).b
              + PSGridGet(src, x, y, z - 1).b) / 5.5f;
  float sc = (PSGridGet(src, x, y, z).c + PSGridGet(src, x, y, z + 1).c
              + PSGridGet(src, x, y, z - 1).c) / 3.3f;
  struct Vec3 out = {sa, sb, sc};
  PSGridEmit(dst, out);
}
"""

_TRIPLE = """
struct Triple { float u; float v; float w; };
DeclareGrid3D(Triple, struct Triple);

void gather_w(const int x, const int y, const int z, PSGrid3DTriple t) {
  float s = PSGridGet(t, x, y, z).u + PSGridGet(t, x + 1, y, z).u
      + PSGridGet(t, x - 1, y, z).u + PSGridGet(t, x, y + 1, z).u
      + PSGridGet(t, x, y - 1, z).u + PSGridGet(t, x, y, z + 1).u
      + PSGridGet(t, x, y, z - 1).u + PSGridGet(t, x, y, z).v
      + PSGridGet(t, x + 1, y, z).v + PSGridGet(t, x - 1, y, z).v
      + PSGridGet(t, x, y + 1, z).v + PSGridGet(t, x, y - 1, z).v
      + PSGridGet(t, x, y, z + 1).v + PSGridGet(t, x, y, z - 1).v;
  PSGridEmitUtype(t.w, s / 14.3);
}

void relax_uv(const int x, const int y, const int z, PSGrid3DTriple t) {
  PSGridEmitUtype(t.u, (PSGridGet(t, x, y, z).u + PSGridGet(t, x, y, z).w) * 0.5);
  PSGridEmitUtype(t.v, (PSGridGet(t, x, y, z).v + PSGridGet(t, x, y, z).w) * 0.5);
}
"""

_PAIR = """
struct Pair { float h[2]; };
DeclareGrid3D(Pair, struct Pair);

void spread(const int x, const int y, const int z, PSGrid3DPair g) {
  float s = PSGridGet(g, x, y, z).h[0] + PSGridGet(g, x - 1, y, z).h[0]
      + PSGridGet(g, x + 1, y, z).h[0] + PSGridGet(g, x, y - 1, z).h[0]
      + PSGridGet(g, x, y + 1, z).h[0] + PSGridGet(g, x, y, z - 1).h[0]
      + PSGridGet(g, x, y, z + 1).h[0];
  PSGridEmitUtype(g.h[1], s);
}
"""

_MULTI = """
struct Cell { float s[2]; float m; float out; };
DeclareGrid3D(Cell, struct Cell);

#define STAR(G, F) (PSGridGet(G, x, y, z).F + PSGridGet(G, x - 1, y, z).F \\
    + PSGridGet(G, x + 1, y, z).F + PSGridGet(G, x, y - 1, z).F \\
    + PSGridGet(G, x, y + 1, z).F + PSGridGet(G, x, y, z - 1).F \\
    + PSGridGet(G, x, y, z + 1).F)

void three_sums(const int x, const int y, const int z, PSGrid3DCell g) {
  float first = STAR(g, s[0]);
  float second = STAR(g, s[1]);
  float third = STAR(g, m);
  PSGridEmitUtype(g.out, first + second + third);
}
"""

_MATRIX = """
struct Mat { float e[3][2]; };
DeclareGrid3D(Mat, struct Mat);

static float star_of(float c, float w, float e, float n, float s, float b, float t) {
  return c + w + e + n + s + b + t;
}

void corners(const int x, const int y, const int z, PSGrid3DMat g) {
  float lo = star_of(PSGridGet(g, x, y, z).e[0][0], PSGridGet(g, x - 1, y, z).e[0][0],
                     PSGridGet(g, x + 1, y, z).e[0][0], PSGridGet(g, x, y - 1, z).e[0][0],
                     PSGridGet(g, x, y + 1, z).e[0][0], PSGridGet(g, x, y, z - 1).e[0][0],
                     PSGridGet(g, x, y, z + 1).e[0][0]);
  float hi = star_of(PSGridGet(g, x, y, z).e[2][1], PSGridGet(g, x - 1, y, z).e[2][1],
                     PSGridGet(g, x + 1, y, z).e[2][1], PSGridGet(g, x, y - 1, z).e[2][1],
                     PSGridGet(g, x, y + 1, z).e[2][1], PSGridGet(g, x, y, z - 1).e[2][1],
                     PSGridGet(g, x, y, z + 1).e[2][1]);
  PSGridEmitUtype(g.e[1][0], lo + hi);
}
"""


def user_cases():
    """name -> dict(src, steps, iters, dtype, init, grids, dump, comps)."""
    import numpy as np
    f4 = np.float32
    return {
        "user-defined-type1": dict(
            src=_VEC3, steps=[("smooth3", [0, 1]), ("smooth3", [1, 0])], iters=5,
            dtype=np.dtype([("a", f4), ("b", f4), ("c", f4)]),
            init=[("a", 0, 0), ("b", 0, 1), ("c", 0, 2)], grids=2, dump=0,
            comps=[("a", 0), ("b", 0), ("c", 0)]),
        "user-defined-type3": dict(
            src=_TRIPLE, steps=[("gather_w", [0]), ("relax_uv", [0])], iters=10,
            dtype=np.dtype([("u", f4), ("v", f4), ("w", f4)]),
            init=[("u", 0, 0), ("v", 0, 1), ("w", 0, None)], grids=1, dump=0,
            comps=[("u", 0), ("v", 0), ("w", 0)]),
        "user-defined-type5": dict(
            src=_PAIR, steps=[("spread", [0])], iters=1,
            dtype=np.dtype([("h", f4, (2,))]), init=[("h", 0, 0), ("h", 1, None)], grids=1,
            dump=0, comps=[("h", 1)]),
        "user-defined-type-multi-members": dict(
            src=_MULTI, steps=[("three_sums", [0])], iters=1,
            dtype=np.dtype([("s", f4, (2,)), ("m", f4), ("out", f4)]),
            init=[("s", 0, 0), ("s", 1, 1), ("m", 0, 2), ("out", 0, None)], grids=1, dump=0,
            comps=[("out", 0)]),
        "user-defined-type-multi-dim-member": dict(
            src=_MATRIX, steps=[("corners", [0])], iters=1,
            dtype=np.dtype([("e", f4, (3, 2))]),
            init=[("e", j * 2 + k, j + k) for j in range(3) for k in range(2)], grids=1, dump=0,
            comps=[("e", 2)]),
    }


def extra_cases():
    """Known-answer cases that only the front end runs (not flat sums, so no
    generic descriptor): name -> case dict in the form of cases.py."""
    n = C.N
    return {
        "15": dict(grids=[(C.PS_FLOAT, (n, n, n))] * 2, init=["ramp", "ramp"],
                   dom=([0, 0, 0], [n, n, n]), run=[([0, 1], -1)], iters=1, dump=1, fmt="%f"),
    }


def _order27():
    out = []
    for dz in (-1, 0, 1):
        for dx, dy in [(0, 0), (1, 0), (-1, 0), (0, 1), (1, 1), (-1, 1), (0, -1), (1, -1),
                       (-1, -1)]:
            out.append((dx, dy, dz))
    return out


def dsl_cases():
    """name -> (source, function, scalars)."""
    out = {
        "7-pt": (_sum_stencil("sum7", "Float", "float", _O7), "sum7", []),
        "7-pt-multi-iterations": (_sum_stencil("sum7", "Float", "float", _O7), "sum7", []),
        "7-pt-double-type": (_sum_stencil("sum7d", "Double", "double", _O7), "sum7d", []),
        "7-pt-int-type": (_sum_stencil("sum7i", "Int", "int", _O7), "sum7i", []),
        "7-pt-periodic": (_sum_stencil("wrap7", "Float", "float", _O7P, True), "wrap7", []),
        "7-pt-neumann-cond": (_NEUMANN, "neumann7", [float(c) for c in C.neumann_coefficients()]),
        "7-pt-type-mix": (_TYPE_MIX, "mixed_types", []),
        "27-pt": (_sum_stencil("box27", "Float", "float", _order27()), "box27", []),
        "27-pt-periodic": (_sum_stencil("wrap27", "Float", "float", _order27(), True), "wrap27",
                           []),
        "asymmetric": (_sum_stencil("skew", "Float", "float",
                                    [(0, 0, 0), (1, 0, 0), (-2, 0, 0)]), "skew", []),
        "asymmetric-periodic": (_ASYM_P, "lopsided", []),
        "stencil-hole": (_sum_stencil("hole", "Float", "float",
                                      [(0, 0, 0), (2, 0, 0), (-2, 0, 0)]), "hole", []),
        "16": (_CLAMPED, "clamped7", []),
        "3-pt-periodic": (_sum_stencil("wrapz", "Float", "float",
                                       [(0, 0, 0), (0, 0, 1), (0, 0, -1)], True), "wrapz", []),
        "3-pt-1d": (_sum_stencil("line3", "Float", "float",
                                 [(-1, 0, 0), (0, 0, 0), (1, 0, 0)], nd=1), "line3", []),
        "9-pt-2d": (_sum_stencil("plane9", "Float", "float",
                                 [(a, b, 0) for a, b in [(0, 0), (-1, 0), (1, 0), (0, -1), (0, 1),
                                                         (-1, -1), (1, -1), (-1, 1), (1, 1)]],
                                 nd=2), "plane9", []),
        "mixed-dim": (_MIXED1, "weighted_x", []),
        "mixed-dim2": (_MIXED2, "weighted_xyz", []),
        "mixed-dim3": (_MIXED3, "weighted_planes", []),
        "redblack": (_inplace_stencil("rb7", _O7, False), "rb7", []),
        "redblack-periodic": (_inplace_stencil("rb7p", _O7, True), "rb7p", []),
        "15": (_BRANCHES, "branches", []),
    }
    return out
