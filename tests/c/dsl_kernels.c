/* A stencil function in the reference's C DSL, for the translator-free front
 * end: `python -m physis_b200.dsl dsl_kernels.c -o libdsl_kernels.so` turns
 * it into an sm_100a kernel library exporting psb_dsl_describe_diffuse. The
 * update is the 7-point diffusion of diffusion3d_physis.c:29-58 with zero-flux
 * faces (a neighbour outside the grid is the point itself). */
#include "physis/physis.h"

void diffuse(const int x, const int y, const int z, PSGrid3DFloat u, PSGrid3DFloat un,
             float ce, float cw, float cn, float cs, float ct, float cb, float cc) {
  const int nx = PSGridDim(u, 0), ny = PSGridDim(u, 1), nz = PSGridDim(u, 2);
  float c = PSGridGet(u, x, y, z);
  float w = x == 0 ? c : PSGridGet(u, x - 1, y, z);
  float e = x == nx - 1 ? c : PSGridGet(u, x + 1, y, z);
  float n = y == 0 ? c : PSGridGet(u, x, y - 1, z);
  float s = y == ny - 1 ? c : PSGridGet(u, x, y + 1, z);
  float b = z == 0 ? c : PSGridGet(u, x, y, z - 1);
  float t = z == nz - 1 ? c : PSGridGet(u, x, y, z + 1);
  PSGridEmit(un, cc * c + cw * w + ce * e + cs * s + cn * n + cb * b + ct * t);
}
