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
    }
    return out
