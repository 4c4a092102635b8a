// FP64 reduction accumulators shared by the grid reduction (k_reduce.cu)
// and the kernel-function reduction (k_generic.cu): SUM with Neumaier
// compensation, PROD in FP64, MAX/MIN exact; fixed shuffle trees, one
// partial per CTA, combined by the last CTA in index order.
#pragma once

#include <cfloat>

#include "device.cuh"

namespace psb {

constexpr int kReduceMaxBlocks = 1184;  // 148 SMs x 8: capacity of the partials

struct RAcc {
  double s;  // value (sum, product, max or min)
  double c;  // compensation (SUM only)
};

__device__ __forceinline__ RAcc racc_init(int op) {
  RAcc a;
  a.c = 0.0;
  switch (op) {
    case PS_MAX: a.s = -DBL_MAX; break;
    case PS_MIN: a.s = DBL_MAX; break;
    case PS_SUM: a.s = 0.0; break;
    default: a.s = 1.0; break;
  }
  return a;
}

// Neumaier step: add x to (s, c).
__device__ __forceinline__ void neumaier(RAcc &a, double x) {
  double t = a.s + x;
  if (fabs(a.s) >= fabs(x)) a.c += (a.s - t) + x;
  else a.c += (x - t) + a.s;
  a.s = t;
}

__device__ __forceinline__ RAcc racc_merge(int op, RAcc a, RAcc b) {
  switch (op) {
    case PS_MAX: a.s = a.s > b.s ? a.s : b.s; return a;
    case PS_MIN: a.s = a.s < b.s ? a.s : b.s; return a;
    case PS_SUM: {
      RAcc r = a;
      neumaier(r, b.s);
      r.c += b.c;
      return r;
    }
    default: a.s = a.s * b.s; return a;
  }
}

__device__ __forceinline__ void racc_add(int op, RAcc &a, double x) {
  switch (op) {
    case PS_MAX: a.s = a.s > x ? a.s : x; break;
    case PS_MIN: a.s = a.s < x ? a.s : x; break;
    case PS_SUM: neumaier(a, x); break;
    default: a.s = a.s * x; break;
  }
}

__device__ __forceinline__ RAcc racc_block(int op, RAcc v, RAcc *scratch) {
  for (int o = 16; o > 0; o >>= 1) {
    RAcc u;
    u.s = __shfl_down_sync(0xffffffffu, v.s, o);
    u.c = __shfl_down_sync(0xffffffffu, v.c, o);
    v = racc_merge(op, v, u);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  RAcc r = racc_init(op);
  if (warp == 0) {
    if (lane < nw) r = scratch[lane];
    for (int o = 16; o > 0; o >>= 1) {
      RAcc u;
      u.s = __shfl_down_sync(0xffffffffu, r.s, o);
      u.c = __shfl_down_sync(0xffffffffu, r.c, o);
      r = racc_merge(op, r, u);
    }
  }
  return r;
}

struct ReduceScratch {
  RAcc *partials;
  unsigned *ticket;
  double *result;
};

// The runtime-owned partials / ticket / result buffer (allocated once).
psb_status reduce_scratch(ReduceScratch *sc);

}  // namespace psb
