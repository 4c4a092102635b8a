// 7-point diffusion kernels (examples/diffusion-benchmark/diffusion3d_physis.c:29-58).
//
//   out = cc*c + cw*w + ce*e + cs*s + cn*n + cb*b + ct*t
//
// evaluated left to right with round-to-nearest multiplies and adds (no
// FMA), so every result is bit-identical to the reference CPU target built
// with -ffp-contract=off.
//
// Two implementations:
//  * k_diff7_plain -- the shape of the reference's generated kernel
//    (translator/cuda_translator.cc:615-907): a 64x4 block, one thread per
//    (x, y), a loop over z, seven global loads per point, branches at the
//    faces. This is the plain one-launch-per-step GPU path.
//  * k_diff7_tma -- the B200 path: each CTA owns a (TX x TY) column of the
//    domain and a chunk of z. Planes of the input, with a one-cell halo in
//    y and a 16-byte halo in x, stream into a ring of shared-memory stages
//    through 3-D TMA tile loads that complete on mbarriers; the z
//    neighbours stay in registers (2.5-D z-streaming), x/y neighbours come
//    from shared memory, and each thread stores 16 bytes at a time. HBM
//    traffic is the compulsory one read and one write per point.
// Clamped faces are resolved with register selects; periodic faces read the
// resident halo of a pitched grid, which every writer keeps current.
#include <algorithm>

#include "k_diffusion7.cuh"

namespace psb {

// --------------------------------------------------------------------------
// Plain kernel
// --------------------------------------------------------------------------
template <typename T, bool PERIODIC>
__global__ void __launch_bounds__(256) k_diff7_plain(GridView in, GridView out, Dom3 d, C7<T> k,
                                                     int images) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x < d.lo[0] || x >= d.hi[0] || y < d.lo[1] || y >= d.hi[1]) return;
  const T *g = (const T *)in.origin;
  T *o = (T *)out.origin;
  const int nx = in.n[0], ny = in.n[1], nz = in.n[2];
  const int64_t sy = in.sy, sz = in.sz;
  for (int z = d.lo[2]; z < d.hi[2]; ++z) {
    const int64_t ci = x + y * sy + z * sz;
    T c = g[ci], w, e, n, s, b, t;
    if (PERIODIC) {
      w = g[(x - 1 + nx) % nx + y * sy + z * sz];
      e = g[(x + 1 + nx) % nx + y * sy + z * sz];
      n = g[x + ((y - 1 + ny) % ny) * sy + z * sz];
      s = g[x + ((y + 1 + ny) % ny) * sy + z * sz];
      b = g[x + y * sy + ((z - 1 + nz) % nz) * sz];
      t = g[x + y * sy + ((z + 1 + nz) % nz) * sz];
    } else {
      if (x == 0) w = c; else w = g[ci - 1];
      if (x == nx - 1) e = c; else e = g[ci + 1];
      if (y == 0) n = c; else n = g[ci - sy];
      if (y == ny - 1) s = c; else s = g[ci + sy];
      if (z == 0) b = c; else b = g[ci - sz];
      if (z == nz - 1) t = c; else t = g[ci + sz];
    }
    T v = diff7_point(k, c, w, e, n, s, b, t);
    o[x + y * out.sy + z * out.sz] = v;
    if (PERIODIC && images) store_face_images(o, out.sy, out.sz, out.n, x, y, z, v);
  }
}

#ifndef PSB_D7_MAXT
#define PSB_D7_MAXT 544
#endif
#ifndef PSB_D7_MINB
#define PSB_D7_MINB 1
#endif
template <typename T, bool PERIODIC, bool FAST>
__global__ void __launch_bounds__(PSB_D7_MAXT, PSB_D7_MINB) k_diff7_tma(const __grid_constant__ CUtensorMap tin,
                                                   GridView out, int nx, int ny, int nz, Dom3 d,
                                                   C7<T> k, TmaGeom geo, int images, int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA destinations must be 128-byte aligned: align the base explicitly
  // (128 spare bytes are allocated for this).
  unsigned char *smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  int b = blockIdx.x;
  const int tile_x = b % geo.tiles_x;
  b /= geo.tiles_x;
  const int tile_y = b % geo.tiles_y;
  const int zc = b / geo.tiles_y;
  diff7_tile<T, PERIODIC, false, FAST>(&tin, out, nx, ny, nz, d, k, geo, tile_x, tile_y, zc,
                                       images, err, smem, nullptr);
}

// --------------------------------------------------------------------------
// Host launchers
// --------------------------------------------------------------------------

template <typename T>
static C7<T> coef_from(const MapImpl &m) {
  // Parameter order of the reference kernel: ce, cw, cn, cs, ct, cb, cc.
  C7<T> k;
  k.ce = (T)m.params[0];
  k.cw = (T)m.params[1];
  k.cn = (T)m.params[2];
  k.cs = (T)m.params[3];
  k.ct = (T)m.params[4];
  k.cb = (T)m.params[5];
  k.cc = (T)m.params[6];
  return k;
}

static Dom3 dom3_of(const MapImpl &m) {
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    d.lo[i] = m.dom.local_min[i];
    d.hi[i] = m.dom.local_max[i];
  }
  return d;
}

template <typename T, bool PERIODIC>
static psb_status launch_plain(MapImpl &m, cudaStream_t s, int64_t *launches) {
  GridImpl *gi = m.grids[0], *go = m.grids[1];
  Dom3 d = dom3_of(m);
  if (d.hi[0] <= d.lo[0] || d.hi[1] <= d.lo[1] || d.hi[2] <= d.lo[2]) return PSB_OK;
  // Launch shape of the reference: block 64x4, grid ceil(max/64) x ceil(max/4).
  dim3 block(64, 4, 1);
  dim3 grid((d.hi[0] + 63) / 64, (d.hi[1] + 3) / 4, 1);
  int images = PERIODIC && go->layout == PSB_LAYOUT_PITCHED;
  k_diff7_plain<T, PERIODIC><<<grid, block, 0, s>>>(gi->view(), go->view(), d, coef_from<T>(m),
                                                     images);
  (*launches)++;
  return PSB_OK;
}

template <typename T, bool PERIODIC, bool FAST>
static psb_status launch_tma(MapImpl &m, const psb_tune_config &cfg, cudaStream_t s,
                             int64_t *launches) {
  constexpr int V = 16 / sizeof(T);
  GridImpl *gi = m.grids[0], *go = m.grids[1];
  Dom3 d = dom3_of(m);
  if (d.hi[0] <= d.lo[0] || d.hi[1] <= d.lo[1] || d.hi[2] <= d.lo[2]) return PSB_OK;
  TmaGeom geo;
  // Consumer threads: tile_x / V along x, tile_y / VY rows; a multiple of 32.
  geo.tx_threads = std::max(1, cfg.tile_x / V);
  geo.ty_threads = std::max(1, cfg.tile_y / kVY);
  while ((geo.tx_threads * geo.ty_threads) % 32) geo.ty_threads++;
  if (geo.tx_threads * geo.ty_threads > 512) return set_status(PSB_ERR_INVALID);
  const int TX = geo.tx_threads * V, TY = geo.ty_threads * kVY;
  geo.bx = TX + 2 * V;
  geo.by = TY + 2;
  if (geo.bx > 256 || geo.by > 256) return set_status(PSB_ERR_INVALID);
  const CUtensorMap *map = nullptr;
  psb_status st = get_tmap(gi, geo.bx, geo.by, &map);
  if (st != PSB_OK) return st;
  geo.ax0 = gi->layout == PSB_LAYOUT_PITCHED ? gi->pad_left : 0;
  geo.ay0 = gi->layout == PSB_LAYOUT_PITCHED ? gi->halo : 0;
  geo.az0 = gi->layout == PSB_LAYOUT_PITCHED ? gi->halo : 0;
  geo.x_base = d.lo[0] / V * V;
  geo.tiles_x = (d.hi[0] - geo.x_base + TX - 1) / TX;
  geo.tiles_y = (d.hi[1] - d.lo[1] + TY - 1) / TY;
  geo.zchunk = std::max(1, cfg.z_chunk);
  int nzc = (d.hi[2] - d.lo[2] + geo.zchunk - 1) / geo.zchunk;
  geo.stages = std::min(std::max(3, cfg.stages), 32);
  geo.stage_bytes = (geo.bx * geo.by * (int)sizeof(T) + 127) / 128 * 128;
  size_t smem = 128 + 512 + (size_t)geo.stages * geo.stage_bytes;
  auto kern = k_diff7_tma<T, PERIODIC, FAST>;
  static size_t configured[2][2][2] = {};
  size_t &conf = configured[sizeof(T) == 8][PERIODIC][FAST];
  if (conf == 0) {
    // Prefer the largest shared-memory carve-out: several CTAs' rings then
    // fit on one SM, which keeps more planes in flight.
    PSB_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    conf = 1;
  }
  if (smem > 48 * 1024 && smem > conf) {
    cudaFuncAttributes fa;
    PSB_TRY(cudaFuncGetAttributes(&fa, kern));
    size_t cap = rt().smem_optin - fa.sharedSizeBytes;
    if (smem > cap) return set_status(PSB_ERR_INVALID);
    PSB_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap));
    conf = cap;
  }
  int64_t nblocks = (int64_t)geo.tiles_x * geo.tiles_y * nzc;
  if (nblocks > 0x7fffffff) return set_status(PSB_ERR_INVALID);
  int images = PERIODIC && go->layout == PSB_LAYOUT_PITCHED;
  const int threads = geo.tx_threads * geo.ty_threads + 32;
  kern<<<(unsigned)nblocks, threads, smem, s>>>(*map, go->view(), gi->pub.dim[0], gi->pub.dim[1],
                                                gi->pub.dim[2], d, coef_from<T>(m), geo, images,
                                                rt().d_error);
  (*launches)++;
  return PSB_OK;
}

// --------------------------------------------------------------------------
// Temporal blocking (two steps per launch), persistent: one CTA per SM
// walks the (tile, z chunk) items blockIdx.x, blockIdx.x + gridDim.x, ...;
// its three rings carry on from item to item.
// --------------------------------------------------------------------------
constexpr int kTbS1 = 6, kTbS2 = 4;  // stages of the input and intermediate rings
constexpr int kTbStage1 = (kTbBX1 * kTbBY1 * 4 + 127) / 128 * 128;
constexpr int kTbStage2 = (kTbBX2 * kTbBY2 * 4 + 127) / 128 * 128;
constexpr int kTbSmem = 128 + 512 + kTbS1 * kTbStage1 + kTbS2 * kTbStage2;

struct TbGeom {
  int ax0, ay0, az0;
  int tiles_x, tiles_y, nzc, zchunk;
  int64_t items;
};

template <bool FAST>
__global__ void __launch_bounds__(kTbThreads, 1) k_diff7_tb2(const __grid_constant__ CUtensorMap tin,
                                                             GridView out, int nx, int ny, int nz,
                                                             C7<float> k, TbGeom tg, int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  const Ring R1{bars, bars + 16, smem + 512, kTbS1, kTbStage1};
  const Ring R2{bars + 32, bars + 48, smem + 512 + kTbS1 * kTbStage1, kTbS2, kTbStage2};
  if (threadIdx.x == 0) {
    ring_init(R1, kTbS1Warps);
    for (int i = 0; i < kTbS2; i++) {
      mbar_init(&R2.full[i], kTbS1Warps);
      mbar_init(&R2.empty[i], kTbS2Warps);
    }
    mbar_fence_init();
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  RingPos p1{0, 0}, p2{0, 0};
  Dom3 d;
  d.lo[0] = d.lo[1] = d.lo[2] = 0;
  d.hi[0] = nx;
  d.hi[1] = ny;
  d.hi[2] = nz;
  TmaGeom g2;  // the intermediate ring, as the ordinary consumer sees it
  g2.tx_threads = 32;
  g2.ty_threads = kTbS2Warps;
  g2.bx = kTbBX2;
  g2.by = kTbBY2;
  g2.stage_bytes = kTbStage2;
  g2.stages = kTbS2;
  g2.ax0 = g2.ay0 = g2.az0 = 0;
  g2.tiles_x = tg.tiles_x;
  g2.tiles_y = tg.tiles_y;
  g2.zchunk = tg.zchunk;
  g2.x_base = 0;
  for (int64_t item = blockIdx.x; item < tg.items; item += gridDim.x) {
    int64_t t = item;
    const int tile_x = (int)(t % tg.tiles_x);
    t /= tg.tiles_x;
    const int tile_y = (int)(t % tg.tiles_y);
    const int zc = (int)(t / tg.tiles_y);
    const int x0 = tile_x * kTbTX, y0 = tile_y * kTbTY, zb = zc * tg.zchunk;
    const int nzl = min(zb + tg.zchunk, nz) - zb;
    bool ok;
    if (warp == 0) {
      if (threadIdx.x != 0) return;
      ok = ring_produce(R1, p1, &tin, (uint32_t)(kTbBX1 * kTbBY1 * 4), x0 - 8 + tg.ax0,
                        y0 - 2 + tg.ay0, zb - 2 + tg.az0, nzl + 4);
      if (!ok) {
        atomicExch(err, 1);
        ring_drain(R1, p1);
        return;
      }
    } else if (warp <= kTbS1Warps) {
      ok = diff7_tb_stage1<FAST>(R1, p1, R2, p2, threadIdx.x - 32, nx, ny, nz, k, x0, y0, zb,
                                 nzl);
      if (!ok) {
        if ((threadIdx.x & 31) == 0) atomicExch(err, 1);
        return;
      }
    } else {
      ok = diff7_consume<float, false, false, FAST>(R2, p2, out, nx, ny, nz, d, k, g2, x0, y0,
                                                    zb, nzl, 0, nullptr,
                                                    threadIdx.x - 32 - 32 * kTbS1Warps);
      if (!ok) {
        if ((threadIdx.x & 31) == 0) atomicExch(err, 1);
        return;
      }
    }
  }
}

// Two steps of the clamped float 7-point map m over the whole grid: reads
// in, writes out (the intermediate step exists only in shared memory). In
// the FMA arithmetic mode both steps use the contracted form, point for
// point as the single-step FMA kernel does.
psb_status diffusion7_tb2_launch(MapImpl &m, GridImpl *in, GridImpl *out, int zchunk,
                                 cudaStream_t s, int64_t *launches) {
  const CUtensorMap *map = nullptr;
  PSB_CHECK(get_tmap(in, kTbBX1, kTbBY1, &map));
  const bool fast = rt().fp_mode == PSB_FP_FMA;
  static bool configured[2] = {false, false};
  if (!configured[fast]) {
    PSB_TRY(cudaFuncSetAttribute(fast ? k_diff7_tb2<true> : k_diff7_tb2<false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, kTbSmem));
    configured[fast] = true;
  }
  TbGeom tg;
  tg.ax0 = in->pad_left;
  tg.ay0 = in->halo;
  tg.az0 = in->halo;
  tg.tiles_x = (in->pub.dim[0] + kTbTX - 1) / kTbTX;
  tg.tiles_y = (in->pub.dim[1] + kTbTY - 1) / kTbTY;
  tg.zchunk = std::max(4, zchunk);
  tg.nzc = (in->pub.dim[2] + tg.zchunk - 1) / tg.zchunk;
  tg.items = (int64_t)tg.tiles_x * tg.tiles_y * tg.nzc;
  C7<float> k{(float)m.params[0], (float)m.params[1], (float)m.params[2], (float)m.params[3],
              (float)m.params[4], (float)m.params[5], (float)m.params[6]};
  const int blocks = (int)std::min<int64_t>(rt().sm_count, tg.items);
  (fast ? k_diff7_tb2<true> : k_diff7_tb2<false>)<<<blocks, kTbThreads, kTbSmem, s>>>(
      *map, out->view(), in->pub.dim[0], in->pub.dim[1], in->pub.dim[2], k, tg, rt().d_error);
  (*launches)++;
  PSB_TRY(cudaGetLastError());
  return PSB_OK;
}

psb_status diffusion7_launch(MapImpl &m, const psb_tune_config &cfg, cudaStream_t s,
                             int64_t *launches) {
  GridImpl *gi = m.grids[0], *go = m.grids[1];
  const bool periodic = m.kernel_id == PSB_KERNEL_DIFFUSION7_PERIODIC;
  const bool dbl = gi->pub.elm_size == 8;
  bool tma = cfg.impl == PSB_IMPL_TMA && tma_eligible(gi) && tma_eligible(go);
  if (tma && periodic) {
    // Periodic TMA reads the input's resident halo.
    tma = gi->layout == PSB_LAYOUT_PITCHED && go->layout == PSB_LAYOUT_PITCHED;
    for (int i = 0; i < 3 && tma; i++)
      if (gi->pub.dim[i] < gi->halo) tma = false;
  }
  if (tma) {
    // The contracted (FMA) arithmetic is a runtime choice (psb_set_fp_mode)
    // of the TMA kernels; the plain kernel always keeps the reference's.
    const bool fast = rt().fp_mode == PSB_FP_FMA;
    psb_status st;
    if (fast)
      st = dbl ? (periodic ? launch_tma<double, true, true>(m, cfg, s, launches)
                           : launch_tma<double, false, true>(m, cfg, s, launches))
               : (periodic ? launch_tma<float, true, true>(m, cfg, s, launches)
                           : launch_tma<float, false, true>(m, cfg, s, launches));
    else
      st = dbl ? (periodic ? launch_tma<double, true, false>(m, cfg, s, launches)
                           : launch_tma<double, false, false>(m, cfg, s, launches))
               : (periodic ? launch_tma<float, true, false>(m, cfg, s, launches)
                           : launch_tma<float, false, false>(m, cfg, s, launches));
    if (st != PSB_ERR_UNSUPPORTED) return st;
  }
  return dbl ? (periodic ? launch_plain<double, true>(m, s, launches)
                         : launch_plain<double, false>(m, s, launches))
             : (periodic ? launch_plain<float, true>(m, s, launches)
                         : launch_plain<float, false>(m, s, launches));
}

}  // namespace psb
