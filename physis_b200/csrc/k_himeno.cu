// Himeno 19-point variable-coefficient Jacobi sweep
// (examples/himeno/himenobmtxpa_physis.c:331-361):
//
//   s0 = a0*p(k+1) + a1*p(j+1) + a2*p(i+1)
//      + b0*(p(j+1,k+1) - p(j-1,k+1) - p(j+1,k-1) + p(j-1,k-1))
//      + b1*(p(i+1,j+1) - p(i+1,j-1) - p(i-1,j+1) + p(i-1,j-1))
//      + b2*(p(i+1,k+1) - p(i+1,k-1) - p(i-1,k+1) + p(i-1,k-1))
//      + c0*p(k-1) + c1*p(j-1) + c2*p(i-1) + wrk1
//   ss = (s0*a3 - p) * bnd
//   p1 = p + omega*ss
//
// (i, j, k) = (x, y, z). Every operation is a round-to-nearest float op in
// the C evaluation order, so results are bit-identical to the reference CPU
// target built without FMA contraction.
//
// The residual sum of ss*ss over the domain (the gosa of the original Himeno
// benchmark) is fused into the sweep: each thread accumulates ss*ss in FP64,
// each CTA reduces its threads in a fixed tree and writes one partial, and
// the last CTA to finish sums the partials in index order into a history
// slot. The result is deterministic and costs no extra pass over memory.
//
// k_himeno_tma streams the pressure field through a ring of shared-memory
// planes loaded by 3-D TMA (box TX+2V by TY+2), like the 7-point kernel; the
// twelve coefficient fields are read once each with 16-byte streaming loads
// issued before the ring wait so they overlap it. k_himeno_plain is the
// reference's generated-kernel shape (thread per (x,y), z loop, global loads).
#include <algorithm>

#include "k_himeno.cuh"

namespace psb {

// Fixed-order block reduction of one double per thread; result in thread 0.
__device__ double block_sum_fixed(double v, double *scratch) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthreads = blockDim.x * blockDim.y;
  const int lane = tid & 31, warp = tid >> 5, nw = (nthreads + 31) >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < nw ? scratch[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;
}

// Write this CTA's partial; the last CTA sums all partials in index order.
__device__ void residual_finish(const Residual &res, double mine, double *scratch) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthreads = blockDim.x * blockDim.y;
  double total = block_sum_fixed(mine, scratch);
  __shared__ int is_last;
  const unsigned bid = blockIdx.x + blockIdx.y * gridDim.x;
  const unsigned nb = gridDim.x * gridDim.y;
  if (tid == 0) {
    res.partials[bid] = total;
    __threadfence();
    unsigned t = atomicAdd(res.ticket, 1u);
    is_last = (t == nb - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double acc = 0.0;
  for (unsigned i = tid; i < nb; i += nthreads) acc += __ldcg(&res.partials[i]);
  double sum = block_sum_fixed(acc, scratch);
  if (tid == 0) {
    unsigned c = *res.counter;
    res.history[c % (unsigned)res.history_len] = sum;
    *res.counter = c + 1;
    *res.ticket = 0;
    __threadfence();
  }
}

// --------------------------------------------------------------------------
// Plain kernel (reference shape, any layout; grids may differ in layout)
// --------------------------------------------------------------------------
struct HimenoViews {
  GridView g[14];  // p_in, p_out, a0 a1 a2 a3 b0 b1 b2 c0 c1 c2 bnd wrk1
};

__global__ void __launch_bounds__(256) k_himeno_plain(HimenoViews v, Dom3 d, float omega,
                                                      Residual res) {
  __shared__ double scratch[32];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const bool active = !(x < d.lo[0] || x >= d.hi[0] || y < d.lo[1] || y >= d.hi[1]);
  double acc = 0.0;
  if (active) {
    const float *p = (const float *)v.g[0].origin;
    const int64_t sy = v.g[0].sy, sz = v.g[0].sz;
    for (int z = d.lo[2]; z < d.hi[2]; ++z) {
      float co[12];
#pragma unroll
      for (int i = 0; i < 12; i++)
        co[i] = ((const float *)v.g[2 + i].origin)[x + y * v.g[2 + i].sy + z * v.g[2 + i].sz];
      auto P = [&](int dx, int dy, int dz) { return p[(x + dx) + (y + dy) * sy + (z + dz) * sz]; };
      float ss;
      float r = himeno_point(co, P(0, 0, 0), P(1, 0, 0), P(-1, 0, 0), P(0, 1, 0), P(0, -1, 0),
                             P(0, 0, 1), P(0, 0, -1), P(0, 1, 1), P(0, -1, 1), P(0, 1, -1),
                             P(0, -1, -1), P(1, 1, 0), P(1, -1, 0), P(-1, 1, 0), P(-1, -1, 0),
                             P(1, 0, 1), P(1, 0, -1), P(-1, 0, 1), P(-1, 0, -1), omega, &ss);
      ((float *)v.g[1].origin)[x + y * v.g[1].sy + z * v.g[1].sz] = r;
      acc += (double)ss * (double)ss;
    }
  }
  if (res.partials) {
    // Linear block id for the partial slot.
    residual_finish(res, acc, scratch);
  }
}

// --------------------------------------------------------------------------
// TMA kernel (all 14 grids share one layout), warp-specialised like the
// 7-point kernel: a producer warp streams pressure planes (box TX+2V by
// TY+2) through a ring of shared-memory stages, consumer warps wait on the
// plane they need and release the one they are done with. Each consumer
// thread owns V = 4 consecutive x points of one row and streams its twelve
// coefficient vectors straight from global memory (read once, 16 bytes
// per load), issued before it waits for the next plane so they overlap.
// --------------------------------------------------------------------------
// Residual of one CTA over its consumer threads (fixed order), then the
// last CTA combines all partials in index order.
__device__ void residual_finish_ws(const Residual &res, double mine, double *scratch, int nct,
                                   int *shared_flag, bool skip) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = nct >> 5;
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
  if (lane == 0) scratch[warp] = mine;
  consumer_bar(nct);
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < nw; w++) t += scratch[w];
    int last = 0;
    if (!skip) {
      res.partials[blockIdx.x] = t;
      __threadfence();
      unsigned k = atomicAdd(res.ticket, 1u);
      last = (k == gridDim.x - 1);
    }
    *shared_flag = last;
  }
  consumer_bar(nct);
  if (!*shared_flag) return;
  __threadfence();
  double acc = 0.0;
  for (unsigned i = tid; i < gridDim.x; i += nct) acc += __ldcg(&res.partials[i]);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  consumer_bar(nct);
  if (lane == 0) scratch[warp] = acc;
  consumer_bar(nct);
  if (tid == 0) {
    double sum = 0.0;
    for (int w = 0; w < nw; w++) sum += scratch[w];
    unsigned c = *res.counter;
    res.history[c % (unsigned)res.history_len] = sum;
    *res.counter = c + 1;
    *res.ticket = 0;
    __threadfence();
  }
}

__global__ void __launch_bounds__(544) k_himeno_tma(const __grid_constant__ CUtensorMap tin,
                                                    float *pout, HimenoCoef cf, int64_t sy,
                                                    int64_t sz, Dom3 d, float omega,
                                                    HimenoGeom geo, Residual res, int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  double *scratch = reinterpret_cast<double *>(smem + 512);   // 17 doubles
  int *flag = reinterpret_cast<int *>(smem + 512 + 8 * 17);    // CTA-wide flags
  if (threadIdx.x == 0) flag[1] = 0;
  int b = blockIdx.x;
  const int tile_x = b % geo.tiles_x;
  b /= geo.tiles_x;
  const int tile_y = b % geo.tiles_y;
  const int zc = b / geo.tiles_y;
  double acc = 0.0;
  bool bad = false;
  // (flag[1] is cleared before the tile's own __syncthreads.)
  const bool consumer = himeno_tile(&tin, pout, cf, sy, sz, d, omega, geo, tile_x, tile_y, zc,
                                    err, smem, &acc, &bad);
  if (!consumer) return;
  if (bad && (threadIdx.x & 31) == 0) atomicExch(&flag[1], 1);
  if (res.partials) {
    // All consumer warps meet here (a timed-out warp too), so the named
    // barriers below always complete.
    const int nct = geo.tx_threads * geo.ty_threads;
    consumer_bar(nct);
    const bool skip = flag[1] != 0;
    residual_finish_ws(res, acc, scratch, nct, &flag[0], skip);
  }
}

// --------------------------------------------------------------------------
// Host launcher
// --------------------------------------------------------------------------
static psb_status ensure_residual(MapImpl &m, int nblocks) {
  if (m.residual_len <= 0) return PSB_OK;
  if (m.partials_cap < nblocks) {
    if (m.d_partials) cudaFree(m.d_partials);
    m.d_partials = nullptr;
    PSB_TRY(cudaMalloc(&m.d_partials, sizeof(double) * nblocks));
    m.partials_cap = nblocks;
  }
  return PSB_OK;
}

psb_status himeno_launch(MapImpl &m, const psb_tune_config &cfg, cudaStream_t s,
                         int64_t *launches) {
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    d.lo[i] = m.dom.local_min[i];
    d.hi[i] = m.dom.local_max[i];
  }
  if (d.hi[0] <= d.lo[0] || d.hi[1] <= d.lo[1] || d.hi[2] <= d.lo[2]) return PSB_OK;
  float omega = (float)m.params[0];
  GridImpl *p0 = m.grids[0];
  bool same = true;
  for (int i = 1; i < 14; i++) {
    GridImpl *g = m.grids[i];
    if (g->layout != p0->layout || g->sy != p0->sy || g->sz != p0->sz ||
        g->origin_off != p0->origin_off)
      same = false;
  }
  bool tma = cfg.impl == PSB_IMPL_TMA && same && tma_eligible(p0);
  Residual res = {nullptr, m.d_ticket, m.d_counter, m.d_history, m.residual_len};
  if (tma) {
    constexpr int V = 4;
    HimenoGeom geo;
    geo.tx_threads = std::max(1, cfg.tile_x / V);
    geo.ty_threads = std::max(1, cfg.tile_y);
    while ((geo.tx_threads * geo.ty_threads) % 32) geo.ty_threads++;
    if (geo.tx_threads * geo.ty_threads > 512) return set_status(PSB_ERR_INVALID);
    const int TX = geo.tx_threads * V, TY = geo.ty_threads;
    geo.bx = TX + 2 * V;
    geo.by = TY + 2;
    const CUtensorMap *map = nullptr;
    psb_status st = get_tmap(p0, geo.bx, geo.by, &map);
    if (st == PSB_OK) {
      geo.ax0 = p0->layout == PSB_LAYOUT_PITCHED ? p0->pad_left : 0;
      geo.ay0 = p0->layout == PSB_LAYOUT_PITCHED ? p0->halo : 0;
      geo.az0 = p0->layout == PSB_LAYOUT_PITCHED ? p0->halo : 0;
      geo.x_base = d.lo[0] / V * V;
      geo.tiles_x = (d.hi[0] - geo.x_base + TX - 1) / TX;
      geo.tiles_y = (d.hi[1] - d.lo[1] + TY - 1) / TY;
      geo.zchunk = std::max(1, cfg.z_chunk);
      geo.stages = std::min(std::max(4, cfg.stages), 32);
      geo.stage_bytes = (geo.bx * geo.by * 4 + 127) / 128 * 128;
      geo.nx = p0->pub.dim[0];
      int nzc = (d.hi[2] - d.lo[2] + geo.zchunk - 1) / geo.zchunk;
      int64_t nblocks = (int64_t)geo.tiles_x * geo.tiles_y * nzc;
      size_t smem = 128 + 768 + (size_t)geo.stages * geo.stage_bytes;
      if (smem <= rt().smem_optin && nblocks < 0x7fffffff) {
        static size_t configured = 0;
        if (smem > 48 * 1024 && smem > configured) {
          // The opt-in limit covers static plus dynamic shared memory.
          cudaFuncAttributes fa;
          PSB_TRY(cudaFuncGetAttributes(&fa, k_himeno_tma));
          size_t cap = rt().smem_optin - fa.sharedSizeBytes;
          if (smem > cap) return set_status(PSB_ERR_INVALID);
          PSB_TRY(cudaFuncSetAttribute(k_himeno_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)cap));
          configured = cap;
        }
        PSB_CHECK(ensure_residual(m, (int)nblocks));
        if (m.residual_len > 0) res.partials = m.d_partials;
        HimenoCoef cf;
        for (int i = 0; i < 12; i++) cf.f[i] = (const float *)m.grids[2 + i]->view().origin;
        const int threads = geo.tx_threads * geo.ty_threads + 32;
        k_himeno_tma<<<(unsigned)nblocks, threads, smem, s>>>(
            *map, (float *)m.grids[1]->view().origin, cf, p0->sy, p0->sz, d, omega, geo, res,
            rt().d_error);
        (*launches)++;
        return PSB_OK;
      }
    }
  }
  HimenoViews v;
  for (int i = 0; i < 14; i++) v.g[i] = m.grids[i]->view();
  dim3 block(64, 4, 1);
  dim3 grid((d.hi[0] + 63) / 64, (d.hi[1] + 3) / 4, 1);
  int nblocks = grid.x * grid.y;
  PSB_CHECK(ensure_residual(m, nblocks));
  if (m.residual_len > 0) res.partials = m.d_partials;
  k_himeno_plain<<<grid, block, 0, s>>>(v, d, omega, res);
  (*launches)++;
  return PSB_OK;
}

}  // namespace psb
