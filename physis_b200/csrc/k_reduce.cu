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
#include <cstdio>
#include <mutex>

#include "reduce.cuh"

namespace psb {

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
    // 64-bit column index: a row may be up to 2^31-1 elements long, and a
    // 32-bit x + 32 would overflow past it.
    for (int64_t x = lane; x < rx; x += 32) racc_add(op, a, (double)row[x]);
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

// (kReduceMaxBlocks, the partials' capacity, is in reduce.cuh.)

psb_status reduce_scratch(ReduceScratch *sc) {
  static void *scratch = nullptr;
  if (!scratch) {
    size_t bytes = sizeof(RAcc) * kReduceMaxBlocks + 256;
    PSB_TRY(cudaMalloc(&scratch, bytes));
    PSB_TRY(cudaMemset(scratch, 0, bytes));
  }
  sc->partials = (RAcc *)scratch;
  sc->ticket = (unsigned *)((char *)scratch + sizeof(RAcc) * kReduceMaxBlocks);
  sc->result = (double *)((char *)scratch + sizeof(RAcc) * kReduceMaxBlocks + 128);
  return PSB_OK;
}

psb_status reduce_view(const GridView &v, int type, int op, const Dom3 &dom, double *result,
                       cudaStream_t s) {
  ReduceScratch sc;
  PSB_CHECK(reduce_scratch(&sc));
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

// ===========================================================================
// Allocation-free reduction entry point.
//
// Some callers cannot call cudaMalloc: a host framework that owns every byte
// of device memory through its own allocator (and counts it against a
// budget), or a latency-critical loop where a cudaMalloc/cudaFree would
// synchronise the device. psb_reduce_noalloc serves them: the same k_reduce
// kernel as psb_reduce, with its per-CTA partials, ticket and result kept in
// the fixed, file-scope device array below instead of a runtime allocation.
//
//  * The array is kNoallocScratchBytes (19,200 bytes); every GPU that loads
//    this library holds it until the process exits.
//  * Host code cannot use the array's name as a device address, so on the
//    first call on each device (with that device current) the address is
//    fetched once with cudaGetSymbolAddress and cached. That first call
//    should therefore come before any stream capture.
//  * Every call shares the array and the array keeps the last call's
//    contents: the ticket is cleared before each launch, and calls that
//    overlap on the GPU (other streams, other host threads) race on it.
//  * The launch never uses more CTAs than the array has partial slots, so
//    the array does not bound the input; extents are bounded by the
//    kernel's 32-bit coordinates (PSB_NOALLOC_MAX_EXTENT per dimension; the
//    column index within a row is 64-bit, so a row of that length does not
//    overflow it) and larger ones are rejected, as are strides whose last
//    element would lie beyond INT64_MAX / 8 elements.
//  * The call blocks: it returns once the result is in host memory. It
//    reads `data` in stream order on `stream`, so the caller orders that
//    stream after whatever last wrote `data` (the runtime's own work runs
//    on a non-blocking stream: psb_sync() before a NULL-stream call).
// ===========================================================================
}  // namespace psb

namespace {
constexpr size_t kNoallocScratchBytes = sizeof(psb::RAcc) * psb::kReduceMaxBlocks + 256;
static_assert(kNoallocScratchBytes == PSB_NOALLOC_SCRATCH_BYTES,
              "PSB_NOALLOC_SCRATCH_BYTES must describe the static scratch array");
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[kNoallocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (set up once).
cudaError_t noalloc_scratch(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNoallocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return cudaSuccess;
}
}  // namespace

extern "C" psb_status psb_reduce_noalloc(const void *data, int type, int op,
                                         const int64_t *extent, const int64_t *stride,
                                         void *stream, double *result) {
  using namespace psb;
  if (!data || !extent || !stride || !result || op < PS_MAX || op > PS_PROD ||
      (type != PS_FLOAT && type != PS_DOUBLE && type != PS_INT && type != PS_LONG)) {
    fprintf(stderr, "psb_reduce_noalloc: invalid argument\n");
    return set_status(PSB_ERR_INVALID);
  }
  for (int i = 0; i < 3; i++) {
    if (extent[i] < 1 || extent[i] > PSB_NOALLOC_MAX_EXTENT) {
      fprintf(stderr,
              "psb_reduce_noalloc: extent[%d] = %lld is outside [1, %lld], the largest "
              "extent this entry point reduces\n",
              i, (long long)extent[i], (long long)PSB_NOALLOC_MAX_EXTENT);
      return set_status(PSB_ERR_INVALID);
    }
  }
  // Rows and planes must not overlap: stride[0] >= nx and stride[1] >=
  // stride[0] * ny, the latter tested as stride[1] / ny >= stride[0] (the
  // same for positive integers) so that no product can overflow. The last
  // element's offset is below nz * stride[1]; bounding that by INT64_MAX / 8
  // keeps every element offset and byte offset representable.
  if (stride[0] < extent[0] || stride[1] / extent[1] < stride[0]) {
    fprintf(stderr, "psb_reduce_noalloc: strides must not overlap rows or planes\n");
    return set_status(PSB_ERR_INVALID);
  }
  if (stride[1] > (INT64_MAX / 8) / extent[2]) {
    fprintf(stderr, "psb_reduce_noalloc: stride[1] * extent[2] exceeds the addressable range\n");
    return set_status(PSB_ERR_INVALID);
  }
  void *scratch = nullptr;
  cudaError_t e = noalloc_scratch(&scratch);
  if (e != cudaSuccess) return cuda_status(e, "psb_reduce_noalloc: cudaGetSymbolAddress");
  cudaStream_t s = (cudaStream_t)stream;
  ReduceScratch sc;
  sc.partials = (RAcc *)scratch;
  sc.ticket = (unsigned *)((char *)scratch + sizeof(RAcc) * kReduceMaxBlocks);
  sc.result = (double *)((char *)scratch + sizeof(RAcc) * kReduceMaxBlocks + 128);
  GridView v;
  v.origin = const_cast<void *>(data);
  v.sy = stride[0];
  v.sz = stride[1];
  v.n[0] = (int)extent[0];
  v.n[1] = (int)extent[1];
  v.n[2] = (int)extent[2];
  v.type = type;
  v.halo = 0;
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    d.lo[i] = 0;
    d.hi[i] = (int)extent[i];
  }
  const int64_t rows = extent[1] * extent[2];
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((rows + 7) / 8, kReduceMaxBlocks));
  // The ticket must start at zero; the array keeps whatever the last call left.
  e = cudaMemsetAsync(sc.ticket, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return cuda_status(e, "psb_reduce_noalloc: clear ticket");
  switch (type) {
    case PS_FLOAT: k_reduce<float><<<blocks, 256, 0, s>>>(v, d, op, sc); break;
    case PS_DOUBLE: k_reduce<double><<<blocks, 256, 0, s>>>(v, d, op, sc); break;
    case PS_INT: k_reduce<int32_t><<<blocks, 256, 0, s>>>(v, d, op, sc); break;
    default: k_reduce<int64_t><<<blocks, 256, 0, s>>>(v, d, op, sc); break;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "psb_reduce_noalloc: launch");
  e = cudaMemcpyAsync(result, sc.result, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "psb_reduce_noalloc: result");
  return PSB_OK;
}
