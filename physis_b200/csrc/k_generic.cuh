// Device-side form of a registered psb_generic_stencil (compact term table,
// bound grids) and the per-point evaluation shared by the map kernel and the
// kernel-function reduction.
#pragma once

#include "device.cuh"

namespace psb {

struct GenFactor {
  int grid;
  int off[3];
  int boundary;
  double c;
};

struct GenTable {
  int nterms;
  int has_post;
  GenFactor post;
  GenFactor a[PSB_MAX_TERMS];
  GenFactor b[PSB_MAX_TERMS];
};

struct GenGrids {
  GridView g[PSB_MAX_GRIDS];
  int axes[PSB_MAX_GRIDS][3];
  int nd[PSB_MAX_GRIDS];
  int out;
};

__device__ __forceinline__ int64_t gen_offset(const GridView &g, const int *axes, int nd,
                                              const GenFactor &f, const int *p) {
  int64_t off = 0;
  for (int k = 0; k < nd; k++) {
    const int ax = axes[k];
    const int n = g.n[k];
    int i = p[ax] + f.off[ax];
    if (f.boundary == PSB_BOUNDARY_PERIODIC) {
      i = (i + n) % n;
    } else if (f.boundary == PSB_BOUNDARY_CLAMP) {
      i = i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
    }
    off += (int64_t)i * (k == 0 ? 1 : (k == 1 ? g.sy : g.sz));
  }
  return off;
}

template <typename A>
__device__ __forceinline__ A gen_factor(const GenGrids &G, const GenFactor &f, const int *p) {
  if (f.grid < 0) return (A)f.c;
  const GridView &g = G.g[f.grid];
  const int64_t o = gen_offset(g, G.axes[f.grid], G.nd[f.grid], f, p);
  switch (g.type) {
    case PS_FLOAT: return (A)((const float *)g.origin)[o];
    case PS_DOUBLE: return (A)((const double *)g.origin)[o];
    case PS_INT: return (A)((const int32_t *)g.origin)[o];
    default: return (A)((const int64_t *)g.origin)[o];
  }
}

template <typename A>
__device__ __forceinline__ void gen_store(const GridView &g, int64_t o, A v) {
  switch (g.type) {
    case PS_FLOAT: ((float *)g.origin)[o] = (float)v; break;
    case PS_DOUBLE: ((double *)g.origin)[o] = (double)v; break;
    case PS_INT: ((int32_t *)g.origin)[o] = (int32_t)v; break;
    default: ((int64_t *)g.origin)[o] = (int64_t)v; break;
  }
}

}  // namespace psb
