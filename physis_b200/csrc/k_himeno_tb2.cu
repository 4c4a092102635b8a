// Himeno Jacobi, two sweeps per pass (temporal blocking of depth 2).
//
// 48 of the 56 compulsory bytes of a Himeno update are the twelve
// coefficient fields (examples/himeno/himenobmtxpa_physis.c:331-361), which
// do not change between sweeps. One pass here advances two sweeps and reads
// each coefficient once: per CTA and tile, a producer thread streams the
// input pressure planes (box TX+8 x TY+4: the tile with a 2-cell halo,
// x rounded out to 16 bytes) into ring R1 and the twelve coefficient planes
// of the tile with a 1-cell halo (box TX+8 x TY+2) into ring RC; five
// "stage-1" warps compute the first sweep over the tile plus a 1-cell halo
// (the points the second sweep reads) into ring R2, whose stages are laid
// out like the coefficient boxes; four "stage-2" warps compute the second
// sweep of the tile from R2 and the same coefficient stages and store it.
// Per output pair of updates the pass moves 4 B of p in, 4 B out and 48 B
// of coefficients (with the halo columns and rows of neighbouring tiles
// mostly from L2): about half the bytes of two single sweeps.
//
// Every point of both sweeps uses the single-sweep arithmetic
// (himeno_point, round-to-nearest, the C evaluation order), and first-sweep
// values outside the domain are the input values (the sweep never writes
// them), so the result equals two single sweeps bit for bit. The residual
// sum of ss*ss of each sweep is accumulated over the tile's own points in
// FP64 and combined per sweep in a fixed order (one partial per CTA, the
// last CTA adds them in index order) into the history of the map whose
// sweep it is.
//
// Persistent: one CTA per SM walks the (tile, z chunk) items blockIdx.x,
// blockIdx.x + gridDim.x, ...; its rings carry on from item to item.
#include <algorithm>
#include <cstring>

#include "k_himeno_tb2.cuh"

namespace psb {

constexpr int kHtThreads = 32 + 32 * (kHtW1 + kHtW2);
constexpr int kHtSmemRing = 1024;  // barriers, scratch and flags before the rings
constexpr int kHtSmem = 128 + kHtSmemRing + kHtRingBytes;

struct HtMaps {
  CUtensorMap coef[12];
};

struct HtGeom {
  int ax0, ay0, az0;  // tensor coordinates of logical (0,0,0)
  int tiles_x, tiles_y, nzc, zchunk;
  int64_t items;
};

__global__ void __launch_bounds__(kHtThreads, 1)
    k_himeno_tb2(const __grid_constant__ CUtensorMap tin, const __grid_constant__ HtMaps cm,
                 float *pout, int64_t sy, int64_t sz, Dom3 d, float omega, HtGeom hg,
                 Residual res1, Residual res2, int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  const HtRings R = ht_rings(reinterpret_cast<uint64_t *>(smem), smem + kHtSmemRing);
  double *scratch = reinterpret_cast<double *>(smem + 512);  // 16 doubles
  int *flags = reinterpret_cast<int *>(smem + 768);          // [0] last CTA, [1] timed out
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    ht_init(R);
    flags[0] = flags[1] = 0;
    mbar_fence_init();
  }
  __syncthreads();

  auto item_geom = [&](int64_t item, int &x0, int &y0, int &zb, int &nzl) {
    int64_t t = item;
    const int tile_x = (int)(t % hg.tiles_x);
    t /= hg.tiles_x;
    const int tile_y = (int)(t % hg.tiles_y);
    const int zc = (int)(t / hg.tiles_y);
    x0 = (d.lo[0] / kHtV * kHtV) + tile_x * kHtTX;
    y0 = d.lo[1] + tile_y * kHtTY;
    zb = d.lo[2] + zc * hg.zchunk;
    nzl = min(zb + hg.zchunk, d.hi[2]) - zb;
  };

  if (warp == 0) {
    if (tid != 0) return;
    tma_prefetch_desc(&tin);
    RingPos p1{0, 0}, pc{0, 0};
    bool ok = true;
    for (int64_t item = blockIdx.x; item < hg.items && ok; item += gridDim.x) {
      int x0, y0, zb, nzl;
      item_geom(item, x0, y0, zb, nzl);
      ok = ht_produce_tile(R, p1, pc, &tin, cm.coef, hg.ax0, hg.ay0, hg.az0, x0, y0, zb, nzl);
    }
    if (!ok) {
      atomicExch(err, 1);
      ht_drain(R, p1, pc);
    }
    return;
  }

  double acc = 0.0;
  bool bad = false;
  if (warp <= kHtW1) {
    RingPos p1{0, 0}, pc{0, 0}, p2{0, 0};
    for (int64_t item = blockIdx.x; item < hg.items && !bad; item += gridDim.x) {
      int x0, y0, zb, nzl;
      item_geom(item, x0, y0, zb, nzl);
      bad = !ht_stage1_tile(R, p1, pc, p2, tid - 32, lane, d, omega, x0, y0, zb, nzl, true, &acc);
    }
  } else {
    RingPos p2{0, 0}, pc{0, 0};
    for (int64_t item = blockIdx.x; item < hg.items && !bad; item += gridDim.x) {
      int x0, y0, zb, nzl;
      item_geom(item, x0, y0, zb, nzl);
      bad = !ht_stage2_tile(R, p2, pc, tid - 32 - 32 * kHtW1, lane, pout, sy, sz, d, omega, x0,
                            y0, zb, nzl, false, true, &acc);
    }
  }

  // ---- residuals: per sweep one partial per CTA (fixed order), the last
  // CTA adds all partials in index order into the sweep's map history. All
  // consumer warps arrive here, a timed-out one too.
  constexpr int nct = 32 * (kHtW1 + kHtW2);
  const int cw = warp - 1;  // consumer warp 0..8
  if (bad && lane == 0) {
    atomicExch(&flags[1], 1);
    atomicExch(err, 1);
  }
  if (!res1.partials) return;
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) scratch[cw] = acc;
  consumer_bar(nct);
  if (tid == 32) {
    double s1 = 0.0, s2 = 0.0;
    for (int w = 0; w < kHtW1; w++) s1 += scratch[w];
    for (int w = kHtW1; w < kHtW1 + kHtW2; w++) s2 += scratch[w];
    int last = 0;
    if (!flags[1]) {
      res1.partials[blockIdx.x] = s1;
      res2.partials[blockIdx.x] = s2;
      __threadfence();
      const unsigned k = atomicAdd(res1.ticket, 1u);
      last = k == gridDim.x - 1;
    }
    flags[0] = last;
  }
  consumer_bar(nct);
  if (!flags[0]) return;
  __threadfence();
  // Consumer warps 0..4 sum sweep 1, warps 5..8 sweep 2.
  const bool first = cw < kHtW1;
  const Residual &RS = first ? res1 : res2;
  const int tg = first ? tid - 32 : tid - 32 - 32 * kHtW1;
  const int ng = first ? 32 * kHtW1 : 32 * kHtW2;
  double s = 0.0;
  for (unsigned i = tg; i < gridDim.x; i += ng) s += __ldcg(&RS.partials[i]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  consumer_bar(nct);
  if (lane == 0) scratch[cw] = s;
  consumer_bar(nct);
  if (tid == 32 || tid == 32 + 32 * kHtW1) {
    double sum = 0.0;
    const int w0 = first ? 0 : kHtW1, w1 = first ? kHtW1 : kHtW1 + kHtW2;
    for (int w = w0; w < w1; w++) sum += scratch[w];
    const unsigned c = *RS.counter;
    RS.history[c % (unsigned)RS.history_len] = sum;
    *RS.counter = c + 1;
    if (first) *res1.ticket = 0;
    __threadfence();
  }
}

// Both maps of PSStencilRun(m1(p0 -> p1), m2(p1 -> p0), n) form a Himeno
// pair the two-sweep pass can advance: pitched float grids of one shape and
// layout, the same coefficient grids, domain and omega.
bool himeno_tb2_pair(MapImpl **ms, int n) {
  if (n != 2) return false;
  const MapImpl &a = *ms[0], &b = *ms[1];
  if (a.kernel_id != PSB_KERNEL_HIMENO19 || b.kernel_id != PSB_KERNEL_HIMENO19) return false;
  if (a.color != -1 || b.color != -1 || a.params[0] != b.params[0]) return false;
  if (b.grids[0] != a.grids[1] || b.grids[1] != a.grids[0] || a.grids[0] == a.grids[1])
    return false;
  if (memcmp(&a.dom, &b.dom, sizeof(a.dom)) != 0) return false;
  for (int i = 2; i < 14; i++)
    if (a.grids[i] != b.grids[i]) return false;
  const GridImpl *g0 = a.grids[0];
  for (int i = 0; i < 14; i++) {
    const GridImpl *g = a.grids[i];
    if (g->layout != PSB_LAYOUT_PITCHED || g->type != PS_FLOAT || !tma_eligible(g) ||
        g->sy != g0->sy || g->sz != g0->sz || g->origin_off != g0->origin_off)
      return false;
    for (int k = 0; k < 3; k++)
      if (g->pub.dim[k] != g0->pub.dim[k]) return false;
  }
  for (int k = 0; k < 3; k++)
    if (a.dom.local_max[k] <= a.dom.local_min[k]) return false;
  // Residual histories: both maps keep one or neither does.
  if ((a.residual_len > 0) != (b.residual_len > 0)) return false;
  return true;
}

static psb_status ht_residual(MapImpl &m, int nblocks, Residual *r) {
  *r = Residual{nullptr, m.d_ticket, m.d_counter, m.d_history, m.residual_len};
  if (m.residual_len <= 0) return PSB_OK;
  if (m.partials_cap < nblocks) {
    if (m.d_partials) cudaFree(m.d_partials);
    m.d_partials = nullptr;
    PSB_TRY(cudaMalloc(&m.d_partials, sizeof(double) * nblocks));
    m.partials_cap = nblocks;
  }
  r->partials = m.d_partials;
  return PSB_OK;
}

// Two sweeps, in -> out: the first is map m1's sweep, the second m2's (their
// residuals go to their histories when both maps have them enabled).
psb_status himeno_tb2_launch(MapImpl &m1, MapImpl &m2, GridImpl *in, GridImpl *out,
                             int zchunk, cudaStream_t s, int64_t *launches) {
  Runtime &r = rt();
  const CUtensorMap *pmap = nullptr;
  PSB_CHECK(get_tmap(in, kHtBX, kHtBY1, &pmap));
  HtMaps cm;
  for (int f = 0; f < 12; f++) {
    const CUtensorMap *c = nullptr;
    PSB_CHECK(get_tmap(m1.grids[2 + f], kHtBX, kHtBY2, &c, CU_TENSOR_MAP_L2_PROMOTION_L2_128B));
    cm.coef[f] = *c;
  }
  static bool configured = false;
  if (!configured) {
    PSB_TRY(cudaFuncSetAttribute(k_himeno_tb2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kHtSmem));
    configured = true;
  }
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    d.lo[i] = m1.dom.local_min[i];
    d.hi[i] = m1.dom.local_max[i];
  }
  HtGeom hg;
  hg.ax0 = in->pad_left;
  hg.ay0 = in->halo;
  hg.az0 = in->halo;
  const int xb = d.lo[0] / kHtV * kHtV;
  hg.tiles_x = (d.hi[0] - xb + kHtTX - 1) / kHtTX;
  hg.tiles_y = (d.hi[1] - d.lo[1] + kHtTY - 1) / kHtTY;
  hg.zchunk = std::max(4, zchunk);
  hg.nzc = (d.hi[2] - d.lo[2] + hg.zchunk - 1) / hg.zchunk;
  hg.items = (int64_t)hg.tiles_x * hg.tiles_y * hg.nzc;
  const int blocks = (int)std::min<int64_t>(r.sm_count, hg.items);
  Residual r1, r2;
  PSB_CHECK(ht_residual(m1, blocks, &r1));
  PSB_CHECK(ht_residual(m2, blocks, &r2));
  if (!r1.partials || !r2.partials) r1.partials = r2.partials = nullptr;  // both or neither
  k_himeno_tb2<<<blocks, kHtThreads, kHtSmem, s>>>(*pmap, cm, (float *)out->view().origin,
                                                   in->sy, in->sz, d, (float)m1.params[0], hg,
                                                   r1, r2, r.d_error);
  (*launches)++;
  PSB_TRY(cudaGetLastError());
  return PSB_OK;
}

}  // namespace psb
