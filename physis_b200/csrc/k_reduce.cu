// Grid reduction (PSReduce / __PSReduceGridFloat / __PSReduceGridDouble).
//
// The reference reduces the whole grid with thrust::reduce / max_element /
// min_element in the element type (runtime/reduce_cuda.h:25-45), allocating
// Thrust temporaries on every call. Here one kernel does it:
//  - each warp walks whole x rows of the domain (coalesced; pitched rows and
//    halo are skipped), each thread accumulates its elements;
//  - SUM accumulates in FP64; for double grids each thread carries a
//    Neumaier compensation term and partial pairs are merged with TwoSum;
//    PROD multiplies in FP64; MAX/MIN are exact in the element type;
//  - threads are combined by a fixed shuffle tree, CTAs write one partial
//    each, and the last CTA to finish (atomic ticket) combines the partials
//    in index order. The order never depends on timing, so a sum is
//    identical from run to run.
// Scratch (partials, ticket, result) lives in a runtime-owned buffer that is
// allocated once.
#include <cfloat>

#include "device.cuh"

namespace psb {

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

__device__ RAcc racc_block(int op, RAcc v, RAcc *scratch) {
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

template <typename T>
__global__ void __launch_bounds__(256) k_reduce(GridView g, Dom3 d, int op, ReduceScratch sc) {
  __shared__ RAcc scratch[32];
  __shared__ int is_last;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int rx = d.hi[0] - d.lo[0], ry = d.hi[1] - d.lo[1];
  const int64_t rows = (int64_t)ry * (d.hi[2] - d.lo[2]);
  const T *base = (const T *)g.origin;
  RAcc a = racc_init(op);
  for (int64_t r = warp; r < rows; r += nwarps) {
    const int y = d.lo[1] + (int)(r % ry);
    const int z = d.lo[2] + (int)(r / ry);
    const T *row = base + (int64_t)y * g.sy + (int64_t)z * g.sz + d.lo[0];
    for (int x = lane; x < rx; x += 32) racc_add(op, a, (double)row[x]);
  }
  RAcc b = racc_block(op, a, scratch);
  if (threadIdx.x == 0) {
    sc.partials[blockIdx.x] = b;
    __threadfence();
    unsigned t = atomicAdd(sc.ticket, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  RAcc acc = racc_init(op);
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
    RAcc p;
    p.s = __ldcg(&sc.partials[i].s);
    p.c = __ldcg(&sc.partials[i].c);
    acc = racc_merge(op, acc, p);
  }
  RAcc tot = racc_block(op, acc, scratch);
  if (threadIdx.x == 0) {
    *sc.result = op == PS_SUM ? tot.s + tot.c : tot.s;
    *sc.ticket = 0;
  }
}

static const int kReduceMaxBlocks = 1184;  // 148 SMs x 8

psb_status reduce_view(const GridView &v, int type, int op, const Dom3 &dom, double *result,
                       cudaStream_t s) {
  static void *scratch = nullptr;
  if (!scratch) {
    size_t bytes = sizeof(RAcc) * kReduceMaxBlocks + 256;
    PSB_TRY(cudaMalloc(&scratch, bytes));
    PSB_TRY(cudaMemset(scratch, 0, bytes));
  }
  ReduceScratch sc;
  sc.partials = (RAcc *)scratch;
  sc.ticket = (unsigned *)((char *)scratch + sizeof(RAcc) * kReduceMaxBlocks);
  sc.result = (double *)((char *)scratch + sizeof(RAcc) * kReduceMaxBlocks + 128);
  int64_t rows = (int64_t)(dom.hi[1] - dom.lo[1]) * (dom.hi[2] - dom.lo[2]);
  if (rows <= 0 || dom.hi[0] <= dom.lo[0]) return set_status(PSB_ERR_INVALID);
  int blocks = (int)std::min<int64_t>((rows + 7) / 8, kReduceMaxBlocks);
  if (blocks < 1) blocks = 1;
  switch (type) {
    case PS_FLOAT: k_reduce<float><<<blocks, 256, 0, s>>>(v, dom, op, sc); break;
    case PS_DOUBLE: k_reduce<double><<<blocks, 256, 0, s>>>(v, dom, op, sc); break;
    case PS_INT: k_reduce<int32_t><<<blocks, 256, 0, s>>>(v, dom, op, sc); break;
    case PS_LONG: k_reduce<int64_t><<<blocks, 256, 0, s>>>(v, dom, op, sc); break;
    default: return set_status(PSB_ERR_INVALID);
  }
  PSB_TRY(cudaMemcpyAsync(result, sc.result, sizeof(double), cudaMemcpyDeviceToHost, s));
  PSB_TRY(cudaStreamSynchronize(s));
  return PSB_OK;
}

}  // namespace psb
