// Seeded synthetic fields generated on the device (benchmarks and tests fill
// tens of GB of grids; generating them on the host would dominate the run).
//
// Element (x, y, z) of a fill with seed s takes the 64-bit hash
// h = splitmix64(s * 0x9E3779B97F4A7C15 + (x + nx*(y + ny*z)))  and
//   kind 0: lo + (hi - lo) * u,  u = (h >> 40) * 2^-24  (uniform [lo, hi))
//   kind 1: lo                                         (constant)
//   kind 2: 1 inside, 0 on the faces                   (Himeno bnd)
//   kind 3: (z / (nz - 1))^2                           (Himeno initial p)
// computed in double and rounded to the grid's type once.
#include <cstring>
#include <mutex>
#include <vector>

#include "device.cuh"

namespace psb {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

template <typename T>
__global__ void k_fill(GridView g, int kind, uint64_t seed, double lo, double hi) {
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t total = (int64_t)nx * ny * nz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const int64_t r = i / nx;
    const int y = (int)(r % ny);
    const int z = (int)(r / ny);
    double v;
    switch (kind) {
      case 0: {
        const uint64_t h = splitmix64(seed * 0x9E3779B97F4A7C15ull + (uint64_t)i);
        v = lo + (hi - lo) * ((double)(h >> 40) * (1.0 / 16777216.0));
        break;
      }
      case 1: v = lo; break;
      case 2:
        v = (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1) ? 0.0 : 1.0;
        break;
      default: {
        const double t = nz > 1 ? (double)z / (double)(nz - 1) : 0.0;
        v = t * t;
        break;
      }
    }
    ((T *)g.origin)[(int64_t)x + (int64_t)y * g.sy + (int64_t)z * g.sz] = (T)v;
  }
}

// Rows of a pitched grid <-> a dense x-fastest array in device memory: one
// warp per row, lanes along x (coalesced on both sides).
template <typename W>
__global__ void __launch_bounds__(256) k_pack(GridView g, W *dense, int unpack) {
  const int nx = g.n[0], ny = g.n[1];
  const int64_t rows = (int64_t)ny * g.n[2];
  const int lane = threadIdx.x & 31;
  for (int64_t r = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5); r < rows;
       r += (int64_t)gridDim.x * 8) {
    const int64_t y = r % ny, z = r / ny;
    W *row = (W *)g.origin + y * g.sy + z * g.sz;
    W *d = dense + r * nx;
    if (unpack)
      for (int x = lane; x < nx; x += 32) row[x] = d[x];
    else
      for (int x = lane; x < nx; x += 32) d[x] = row[x];
  }
}

static std::mutex g_stage_mu;
static cudaMemPool_t g_stage_pool = nullptr;

static cudaMemPool_t staging_pool() {
  std::lock_guard<std::mutex> lk(g_stage_mu);
  if (!g_stage_pool) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = rt().device;
    if (cudaMemPoolCreate(&g_stage_pool, &props) != cudaSuccess) {
      cudaGetLastError();
      g_stage_pool = nullptr;
      return nullptr;
    }
    // Keep up to 1 GB of staging memory between copies.
    uint64_t keep = 1ull << 30;
    cudaMemPoolSetAttribute(g_stage_pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  return g_stage_pool;
}

// Host <-> pitched grid on stream s. The copy engines move a strided 3-D copy
// row by row, which is slow for the short rows of narrow grids; instead the
// dense host array crosses the link as one contiguous block into a staging
// buffer (stream-ordered pool, no device-wide synchronisation) and k_pack
// moves it into (or out of) the rows at HBM speed. If no staging memory can
// be had, the strided copy is used.
psb_status pitched_transfer(GridImpl *g, void *host, bool h2d, cudaStream_t s) {
  const int E = g->pub.elm_size;
  const size_t bytes = (size_t)g->pub.num_elms * E;
  const GridView v = g->view();
  void *stage = nullptr;
  cudaMemPool_t pool = staging_pool();
  if (pool && cudaMallocFromPoolAsync(&stage, bytes, pool, s) == cudaSuccess) {
    const int64_t rows = (int64_t)v.n[1] * v.n[2];
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((rows + 7) / 8,
                                                                    (int64_t)rt().sm_count * 16));
    if (h2d) PSB_TRY(cudaMemcpyAsync(stage, host, bytes, cudaMemcpyHostToDevice, s));
    if (E == 4)
      k_pack<uint32_t><<<blocks, 256, 0, s>>>(v, (uint32_t *)stage, h2d ? 1 : 0);
    else
      k_pack<uint64_t><<<blocks, 256, 0, s>>>(v, (uint64_t *)stage, h2d ? 1 : 0);
    PSB_TRY(cudaGetLastError());
    if (!h2d) PSB_TRY(cudaMemcpyAsync(host, stage, bytes, cudaMemcpyDeviceToHost, s));
    PSB_TRY(cudaFreeAsync(stage, s));
    return PSB_OK;
  }
  cudaGetLastError();
  const int nx = v.n[0], ny = v.n[1], nz = v.n[2];
  const int nd = g->pub.num_dims;
  cudaMemcpy3DParms p;
  memset(&p, 0, sizeof(p));
  cudaPitchedPtr dense = make_cudaPitchedPtr(host, (size_t)nx * E, nx, ny);
  cudaPitchedPtr dev = make_cudaPitchedPtr(g->alloc, (size_t)g->pitch * E, g->pitch, g->rows);
  cudaPos pos = make_cudaPos((size_t)g->pad_left * E, nd > 1 ? g->halo : 0, nd > 2 ? g->halo : 0);
  if (h2d) {
    p.srcPtr = dense;
    p.dstPtr = dev;
    p.dstPos = pos;
    p.kind = cudaMemcpyHostToDevice;
  } else {
    p.srcPtr = dev;
    p.srcPos = pos;
    p.dstPtr = dense;
    p.kind = cudaMemcpyDeviceToHost;
  }
  p.extent = make_cudaExtent((size_t)nx * E, ny, nz);
  PSB_TRY(cudaMemcpy3DAsync(&p, s));
  return PSB_OK;
}

// User-defined point types: a host array of records <-> one pitched grid per
// scalar component. One thread per point walks the record's components, so
// the record is read (or written) contiguously and every component grid is
// written (or read) coalesced across the warp.
struct AosComp {
  GridView v;
  int offset;  // bytes into the record
  int esize;   // 4 or 8
};

__global__ void __launch_bounds__(256) k_aos(const AosComp *comps, int ncomp, int record,
                                             unsigned char *stage, int64_t npts, int unpack) {
  const GridView v0 = comps[0].v;
  const int nx = v0.n[0], ny = v0.n[1];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npts;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const int64_t r = i / nx;
    const int64_t y = r % ny, z = r / ny;
    unsigned char *rec = stage + i * record;
    for (int c = 0; c < ncomp; c++) {
      const AosComp &a = comps[c];
      const int64_t o = x + y * a.v.sy + z * a.v.sz;
      if (a.esize == 4) {
        uint32_t *g = (uint32_t *)a.v.origin + o;
        uint32_t *h = (uint32_t *)(rec + a.offset);
        if (unpack) *g = *h; else *h = *g;
      } else {
        uint64_t *g = (uint64_t *)a.v.origin + o;
        uint64_t *h = (uint64_t *)(rec + a.offset);
        if (unpack) *g = *h; else *h = *g;
      }
    }
  }
}

psb_status user_transfer(GridImpl *g, void *host, bool h2d, cudaStream_t s) {
  const psb_user_type &ut = g->utype;
  std::vector<AosComp> comps;
  for (int f = 0; f < ut.nfields; f++)
    for (int k = 0; k < ut.field_count[f]; k++) {
      AosComp a;
      GridImpl *c = g->comps[g->comp_field_first[f] + k];
      a.v = c->view();
      a.esize = c->pub.elm_size;
      a.offset = (int)(ut.field_offset[f] + (size_t)k * a.esize);
      comps.push_back(a);
    }
  const int64_t npts = g->pub.num_elms;
  const size_t data = (size_t)npts * ut.record_bytes;
  const size_t table = comps.size() * sizeof(AosComp);
  const size_t data_off = (table + 255) / 256 * 256;
  cudaMemPool_t pool = staging_pool();
  if (!pool) return set_status(PSB_ERR_NOMEM);
  void *stage = nullptr;
  PSB_TRY(cudaMallocFromPoolAsync(&stage, data_off + data, pool, s));
  unsigned char *base = (unsigned char *)stage;
  PSB_TRY(cudaMemcpyAsync(base, comps.data(), table, cudaMemcpyHostToDevice, s));
  if (h2d) PSB_TRY(cudaMemcpyAsync(base + data_off, host, data, cudaMemcpyHostToDevice, s));
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((npts + 255) / 256,
                                                                  (int64_t)rt().sm_count * 16));
  k_aos<<<blocks, 256, 0, s>>>((const AosComp *)base, (int)comps.size(), (int)ut.record_bytes,
                               base + data_off, npts, h2d ? 1 : 0);
  PSB_TRY(cudaGetLastError());
  if (!h2d) PSB_TRY(cudaMemcpyAsync(host, base + data_off, data, cudaMemcpyDeviceToHost, s));
  PSB_TRY(cudaFreeAsync(stage, s));
  return PSB_OK;
}

// Two-phase copy-out for callers that overlap the transfer with kernels
// occupying every SM: pack into a staging buffer on stream s (a short HBM
// pass), then move the dense block to the host on another stream after an
// event (copy engines only) and release the buffer there.
psb_status pitched_stage_out(GridImpl *g, void **stage, cudaStream_t s) {
  const int E = g->pub.elm_size;
  const size_t bytes = (size_t)g->pub.num_elms * E;
  const GridView v = g->view();
  *stage = nullptr;
  cudaMemPool_t pool = staging_pool();
  if (!pool) return set_status(PSB_ERR_NOMEM);
  PSB_TRY(cudaMallocFromPoolAsync(stage, bytes, pool, s));
  const int64_t rows = (int64_t)v.n[1] * v.n[2];
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((rows + 7) / 8,
                                                                  (int64_t)rt().sm_count * 16));
  if (E == 4)
    k_pack<uint32_t><<<blocks, 256, 0, s>>>(v, (uint32_t *)*stage, 0);
  else
    k_pack<uint64_t><<<blocks, 256, 0, s>>>(v, (uint64_t *)*stage, 0);
  PSB_TRY(cudaGetLastError());
  return PSB_OK;
}

}  // namespace psb

using namespace psb;

extern "C" psb_status psb_grid_fill(__PSGrid *p, int kind, uint64_t seed, double lo, double hi) {
  GridImpl *g = as_impl(p);
  if (!g || g->user_type || !g->comps.empty() || kind < 0 || kind > 3)
    return set_status(PSB_ERR_INVALID);
  PSB_CHECK(ensure_init());
  Runtime &r = rt();
  GridView v = g->view();
  const int64_t total = (int64_t)v.n[0] * v.n[1] * v.n[2];
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)r.sm_count * 16);
  switch (g->type) {
    case PS_FLOAT: k_fill<float><<<blocks, 256, 0, r.stream>>>(v, kind, seed, lo, hi); break;
    case PS_DOUBLE: k_fill<double><<<blocks, 256, 0, r.stream>>>(v, kind, seed, lo, hi); break;
    case PS_INT: k_fill<int32_t><<<blocks, 256, 0, r.stream>>>(v, kind, seed, lo, hi); break;
    case PS_LONG: k_fill<int64_t><<<blocks, 256, 0, r.stream>>>(v, kind, seed, lo, hi); break;
    default: return set_status(PSB_ERR_INVALID);
  }
  PSB_TRY(cudaGetLastError());
  if (g->layout == PSB_LAYOUT_PITCHED) g->ghost_valid = PSB_BOUNDARY_NONE;
  return PSB_OK;
}
