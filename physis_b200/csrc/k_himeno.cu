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

#include "device.cuh"

namespace psb {

struct HimenoCoef {
  const float *f[12];  // a0 a1 a2 a3 b0 b1 b2 c0 c1 c2 bnd wrk1 (origins)
};

struct Residual {
  double *partials;   // one per CTA, or nullptr when disabled
  unsigned *ticket;
  unsigned *counter;
  double *history;
  int history_len;
};

__device__ __forceinline__ float himeno_point(const float *co, float pc, float pxp, float pxm,
                                              float pyp, float pym, float pzp, float pzm,
                                              float pypzp, float pymzp, float pypzm, float pymzm,
                                              float pxpyp, float pxpym, float pxmyp, float pxmym,
                                              float pxpzp, float pxpzm, float pxmzp, float pxmzm,
                                              float omega, float *ss_out) {
  // co: a0 a1 a2 a3 b0 b1 b2 c0 c1 c2 bnd wrk1 at this point.
  float s0 = xmul(co[0], pzp);
  s0 = xadd(s0, xmul(co[1], pyp));
  s0 = xadd(s0, xmul(co[2], pxp));
  s0 = xadd(s0, xmul(co[4], xadd(xsub(xsub(pypzp, pymzp), pypzm), pymzm)));
  s0 = xadd(s0, xmul(co[5], xadd(xsub(xsub(pxpyp, pxpym), pxmyp), pxmym)));
  s0 = xadd(s0, xmul(co[6], xadd(xsub(xsub(pxpzp, pxpzm), pxmzp), pxmzm)));
  s0 = xadd(s0, xmul(co[7], pzm));
  s0 = xadd(s0, xmul(co[8], pym));
  s0 = xadd(s0, xmul(co[9], pxm));
  s0 = xadd(s0, co[11]);
  float ss = xmul(xsub(xmul(s0, co[3]), pc), co[10]);
  *ss_out = ss;
  return xadd(pc, xmul(omega, ss));
}

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
struct HimenoGeom {
  int ax0, ay0, az0;
  int tiles_x, tiles_y, zchunk, stages, bx, by, stage_bytes, x_base;
  int nx;          // row length, bounds the 16-byte coefficient loads
  int tx_threads;  // consumer threads along x (TX / V)
  int ty_threads;  // consumer rows (TY)
};

__device__ __forceinline__ void consumer_bar(int nct) {
  asm volatile("bar.sync 1, %0;" ::"r"(nct) : "memory");
}

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
  constexpr int V = 4;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *empty = full + 32;
  double *scratch = reinterpret_cast<double *>(smem + 512);   // 17 doubles
  int *flag = reinterpret_cast<int *>(smem + 512 + 8 * 17);    // CTA-wide flags
  unsigned char *ring = smem + 768;

  const int S = geo.stages;
  const int nct = geo.tx_threads * geo.ty_threads;
  const int ncw = nct >> 5;
  const int TX = geo.tx_threads * V, TY = geo.ty_threads;
  int b = blockIdx.x;
  const int tile_x = b % geo.tiles_x;
  b /= geo.tiles_x;
  const int tile_y = b % geo.tiles_y;
  const int zc = b / geo.tiles_y;
  const int x0 = geo.x_base + tile_x * TX;
  const int y0 = d.lo[1] + tile_y * TY;
  const int zb = d.lo[2] + zc * geo.zchunk;
  const int ze = min(zb + geo.zchunk, d.hi[2]);
  const int nzl = ze - zb;
  const int np = nzl + 2;
  const int tid = threadIdx.x;

  if (tid == 0) {
    for (int i = 0; i < S; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], ncw);
    }
    flag[1] = 0;
    mbar_fence_init();
  }
  __syncthreads();

  if (tid >= nct) {
    if (tid != nct) return;
    tma_prefetch_desc(&tin);
    const uint32_t bytes = (uint32_t)(geo.bx * geo.by * sizeof(float));
    int slot = 0, round = 0, issued = 0;
    bool ok = true;
    for (int j = 0; j < np; j++) {
      if (round > 0 && !mbar_wait_bounded(&empty[slot], (round - 1) & 1)) {
        ok = false;
        break;
      }
      mbar_arrive_expect_tx(&full[slot], bytes);
      tma_load_3d(ring + slot * geo.stage_bytes, &tin, &full[slot], x0 - V + geo.ax0,
                  y0 - 1 + geo.ay0, zb - 1 + j + geo.az0);
      issued++;
      if (++slot == S) {
        slot = 0;
        round++;
      }
    }
    if (!ok) {
      atomicExch(err, 1);
      for (int j = 0; j < issued; j++) {
        long long t0 = clock64();
        while (!mbar_try_wait(&full[j % S], (j / S) & 1) && clock64() - t0 < 200000000LL) {
        }
      }
    }
    return;
  }

  // ---------------- consumers ----------------
  const int tx = tid % geo.tx_threads, ty = tid / geo.tx_threads;
  const int lane = tid & 31;
  const int BX = geo.bx;
  const int rc = (ty + 1) * BX + V + tx * V;
  const int xg0 = x0 + tx * V;
  const int yg = y0 + ty;
  const bool row_in = yg >= d.lo[1] && yg < d.hi[1];
  const bool vec_ok = xg0 + V <= geo.nx;
  const bool xvec = xg0 >= d.lo[0] && xg0 + V <= d.hi[0];
  auto wait_plane = [&](int slot, int round) -> bool {
    bool ok = mbar_wait_bounded(&full[slot], round & 1);
    return __all_sync(0xffffffffu, ok);
  };
  auto plane_ptr = [&](int slot) -> const float * {
    return reinterpret_cast<const float *>(ring + slot * geo.stage_bytes);
  };
  double acc = 0.0;
  bool bad = !wait_plane(0, 0);
  bad = bad || !wait_plane(1 % S, 1 / S);
  int s_m = 0, s_c = 1 % S;        // slots of planes z-1 and z
  int s_p = 1 % S, r_p = 0;        // slot / round of plane z+1 (advanced before use)
  int64_t off = (int64_t)xg0 + (int64_t)yg * sy + (int64_t)zb * sz;
  for (int jj = 0; jj < nzl && !bad; jj++) {
    const int z = zb + jj;
    float co[12][V];
    if (row_in) {
#pragma unroll
      for (int i = 0; i < 12; i++) {
        if (vec_ok) {
          Vec16<float> q = ldg16_stream(cf.f[i] + off);
#pragma unroll
          for (int v = 0; v < V; v++) co[i][v] = q.v[v];
        } else {
#pragma unroll
          for (int v = 0; v < V; v++) co[i][v] = xg0 + v < geo.nx ? cf.f[i][off + v] : 0.f;
        }
      }
    }
    if (++s_p == S) {
      s_p = 0;
      r_p++;
    }
    if (!wait_plane(s_p, r_p)) {
      bad = true;
      break;
    }
    const float *pm = plane_ptr(s_m), *pc = plane_ptr(s_c), *pp = plane_ptr(s_p);
    if (row_in) {
      float outv[V];
#pragma unroll
      for (int v = 0; v < V; v++) {
        const int o = rc + v;
        float c[12];
#pragma unroll
        for (int i = 0; i < 12; i++) c[i] = co[i][v];
        float ss;
        outv[v] = himeno_point(c, pc[o], pc[o + 1], pc[o - 1], pc[o + BX], pc[o - BX], pp[o],
                               pm[o], pp[o + BX], pp[o - BX], pm[o + BX], pm[o - BX],
                               pc[o + 1 + BX], pc[o + 1 - BX], pc[o - 1 + BX], pc[o - 1 - BX],
                               pp[o + 1], pm[o + 1], pp[o - 1], pm[o - 1], omega, &ss);
        if (xg0 + v >= d.lo[0] && xg0 + v < d.hi[0]) acc += (double)ss * (double)ss;
      }
      float *dst = pout + off;
      if (xvec) {
        *reinterpret_cast<float4 *>(dst) = make_float4(outv[0], outv[1], outv[2], outv[3]);
      } else {
#pragma unroll
        for (int v = 0; v < V; v++)
          if (xg0 + v >= d.lo[0] && xg0 + v < d.hi[0]) dst[v] = outv[v];
      }
    }
    // Plane z-1 is done for this warp.
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s_m]);
    s_m = s_c;
    s_c = s_p;
    off += sz;
    (void)z;
  }
  if (bad) {
    if (lane == 0) {
      atomicExch(err, 1);
      atomicExch(&flag[1], 1);
    }
  }
  if (res.partials) {
    // All consumer warps meet here (a timed-out warp too), so the named
    // barriers below always complete.
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
