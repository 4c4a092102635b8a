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

#include "k_himeno.cuh"

namespace psb {

constexpr int kHtTX = 64, kHtTY = 8, kHtV = 4;
constexpr int kHtBX = kHtTX + 8;           // every box: x from x0 - 4, 16-byte aligned
constexpr int kHtBY1 = kHtTY + 4;          // input p: y from y0 - 2
constexpr int kHtBY2 = kHtTY + 2;          // first sweep and coefficients: y from y0 - 1
constexpr int kHtS1 = 6, kHtS2 = 4, kHtSC = 4;
constexpr int kHtStage1 = (kHtBX * kHtBY1 * 4 + 127) / 128 * 128;
constexpr int kHtStage2 = (kHtBX * kHtBY2 * 4 + 127) / 128 * 128;
constexpr int kHtField = kHtStage2;        // one coefficient box
constexpr int kHtStageC = 12 * kHtField;
constexpr int kHtW1 = 5, kHtW2 = 4;        // stage-1 and stage-2 warps
constexpr int kHtThreads = 32 + 32 * (kHtW1 + kHtW2);
constexpr int kHtSmemRing = 1024;          // barriers and scratch before the rings
constexpr int kHtSmem = 128 + kHtSmemRing + kHtS1 * kHtStage1 + kHtS2 * kHtStage2 +
                        kHtSC * kHtStageC;
static_assert(kHtTX / kHtV * (kHtTY + 2) == 32 * kHtW1, "stage-1 threads cover the halo rows");
static_assert(kHtTX / kHtV * kHtTY == 32 * kHtW2, "stage-2 threads cover the tile");

struct HtMaps {
  CUtensorMap coef[12];
};

struct HtGeom {
  int ax0, ay0, az0;            // tensor coordinates of logical (0,0,0)
  int tiles_x, tiles_y, nzc, zchunk;
  int64_t items;
};

// 19 pressure values around offset o of three planes laid out with row
// length kHtBX (m: z-1, c: z, p: z+1) and the point's 12 coefficients.
__device__ __forceinline__ float ht_point(const float *co, const float *qm, const float *qc,
                                          const float *qp, int o, float omega, float *ss) {
  constexpr int B = kHtBX;
  return himeno_point(co, qc[o], qc[o + 1], qc[o - 1], qc[o + B], qc[o - B], qp[o], qm[o],
                      qp[o + B], qp[o - B], qm[o + B], qm[o - B], qc[o + 1 + B], qc[o + 1 - B],
                      qc[o - 1 + B], qc[o - 1 - B], qp[o + 1], qm[o + 1], qp[o - 1], qm[o - 1],
                      omega, ss);
}

__device__ __forceinline__ bool ht_wait(uint64_t *bar, uint32_t parity) {
  const bool ok = mbar_wait_bounded(bar, parity);
  return __all_sync(0xffffffffu, ok);
}

__device__ __forceinline__ void ht_release(uint64_t *bar, int lane) {
  __syncwarp();
  if (lane == 0) mbar_arrive(bar);
}

__global__ void __launch_bounds__(kHtThreads, 1)
    k_himeno_tb2(const __grid_constant__ CUtensorMap tin, const __grid_constant__ HtMaps cm,
                 float *pout, int64_t sy, int64_t sz, Dom3 d, float omega, HtGeom hg,
                 Residual res1, Residual res2, int *err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  // full/empty barriers: R1 at 0/8, R2 at 16/24, RC at 32/40 (8 each).
  uint64_t *f1 = bars, *e1 = bars + 8, *f2 = bars + 16, *e2 = bars + 24, *fc = bars + 32,
           *ec = bars + 40;
  double *scratch = reinterpret_cast<double *>(smem + 512);  // 16 doubles
  int *flags = reinterpret_cast<int *>(smem + 768);          // [0] last CTA, [1] timed out
  unsigned char *r1 = smem + kHtSmemRing;
  unsigned char *r2 = r1 + kHtS1 * kHtStage1;
  unsigned char *rc = r2 + kHtS2 * kHtStage2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int i = 0; i < kHtS1; i++) {
      mbar_init(&f1[i], 1);
      mbar_init(&e1[i], kHtW1);
    }
    for (int i = 0; i < kHtS2; i++) {
      mbar_init(&f2[i], kHtW1);
      mbar_init(&e2[i], kHtW2);
    }
    for (int i = 0; i < kHtSC; i++) {
      mbar_init(&fc[i], 1);
      mbar_init(&ec[i], kHtW1 + kHtW2);
    }
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
    // ---- producer: input planes zb-2 .. zb+nzl+1 into R1 and coefficient
    // planes zb-1 .. zb+nzl into RC, each RC plane issued after the R1 plane
    // that the first sweep needs with it.
    if (tid != 0) return;
    tma_prefetch_desc(&tin);
    RingPos p1{0, 0}, pc{0, 0};
    bool ok = true;
    auto put1 = [&](int x0, int y0, int z) -> bool {
      if (p1.round > 0 && !mbar_wait_bounded(&e1[p1.slot], (p1.round - 1) & 1)) return false;
      mbar_arrive_expect_tx(&f1[p1.slot], (uint32_t)(kHtBX * kHtBY1 * 4));
      tma_load_3d(r1 + p1.slot * kHtStage1, &tin, &f1[p1.slot], x0 - 4 + hg.ax0,
                  y0 - 2 + hg.ay0, z + hg.az0);
      ring_next(p1, kHtS1);
      return true;
    };
    auto putc = [&](int x0, int y0, int z) -> bool {
      if (pc.round > 0 && !mbar_wait_bounded(&ec[pc.slot], (pc.round - 1) & 1)) return false;
      mbar_arrive_expect_tx(&fc[pc.slot], (uint32_t)(12 * kHtBX * kHtBY2 * 4));
      unsigned char *dst = rc + pc.slot * kHtStageC;
      for (int f = 0; f < 12; f++)
        tma_load_3d(dst + f * kHtField, &cm.coef[f], &fc[pc.slot], x0 - 4 + hg.ax0,
                    y0 - 1 + hg.ay0, z + hg.az0);
      ring_next(pc, kHtSC);
      return true;
    };
    for (int64_t item = blockIdx.x; item < hg.items && ok; item += gridDim.x) {
      int x0, y0, zb, nzl;
      item_geom(item, x0, y0, zb, nzl);
      ok = put1(x0, y0, zb - 2) && put1(x0, y0, zb - 1);
      for (int j = 0; j < nzl + 2 && ok; j++)
        ok = put1(x0, y0, zb + j) && putc(x0, y0, zb - 1 + j);
    }
    if (!ok) {
      atomicExch(err, 1);
      ring_drain(Ring{f1, e1, r1, kHtS1, kHtStage1}, p1);
      ring_drain(Ring{fc, ec, rc, kHtSC, kHtStageC}, pc);
    }
    return;
  }

  double acc = 0.0;
  bool bad = false;
  if (warp <= kHtW1) {
    // ---- stage 1: the first sweep over the tile and a 1-cell halo. Thread
    // t owns 4 x points of halo row t / 16 (y0 - 1 + row); every eighth
    // thread also owns one of the 20 edge points (x0 - 1 and x0 + TX of
    // each row).
    const int t = tid - 32;
    const int tx = t % (kHtTX / kHtV), row = t / (kHtTX / kHtV);
    const int cofs = row * kHtBX + 4 + tx * kHtV;        // R2 / RC offset of the vector
    const int pofs = (row + 1) * kHtBX + 4 + tx * kHtV;  // R1 offset of the vector
    const bool edge = (t & 7) == 0;
    const int e = t >> 3;                                // 0..19
    const int ecol = e / (kHtTY + 2), erow = e % (kHtTY + 2);
    const int ex_off = ecol ? 4 + kHtTX : 3;
    const int ecofs = erow * kHtBX + ex_off, epofs = (erow + 1) * kHtBX + ex_off;
    RingPos p1{0, 0}, pc{0, 0}, p2{0, 0};
    for (int64_t item = blockIdx.x; item < hg.items && !bad; item += gridDim.x) {
      int x0, y0, zb, nzl;
      item_geom(item, x0, y0, zb, nzl);
      const int xg = x0 + tx * kHtV, yg = y0 - 1 + row;
      const int ex = ecol ? x0 + kHtTX : x0 - 1, ey = y0 - 1 + erow;
      const bool row_in = yg >= d.lo[1] && yg < d.hi[1];
      const bool row_own = row_in && row >= 1 && row <= kHtTY;
      RingPos pm = p1, pz = p1;  // planes z-1 and z of the input
      ring_next(pz, kHtS1);
      RingPos pp = pz;
      bad = !ht_wait(&f1[pm.slot], pm.round & 1) || !ht_wait(&f1[pz.slot], pz.round & 1);
      for (int j = 0; j < nzl + 2 && !bad; j++) {
        const int z = zb - 1 + j;
        ring_next(pp, kHtS1);
        if (!ht_wait(&f1[pp.slot], pp.round & 1) || !ht_wait(&fc[pc.slot], pc.round & 1)) {
          bad = true;
          break;
        }
        const float *qm = reinterpret_cast<const float *>(r1 + pm.slot * kHtStage1);
        const float *qc = reinterpret_cast<const float *>(r1 + pz.slot * kHtStage1);
        const float *qp = reinterpret_cast<const float *>(r1 + pp.slot * kHtStage1);
        const unsigned char *cs = rc + pc.slot * kHtStageC;
        const bool z_in = z >= d.lo[2] && z < d.hi[2];
        const bool z_own = z_in && j >= 1 && j <= nzl;
        float outv[kHtV];
        {
          Vec16<float> co[12];
#pragma unroll
          for (int f = 0; f < 12; f++)
            co[f] = lds16(reinterpret_cast<const float *>(cs + f * kHtField) + cofs);
#pragma unroll
          for (int v = 0; v < kHtV; v++) {
            const int x = xg + v;
            float c[12];
#pragma unroll
            for (int f = 0; f < 12; f++) c[f] = co[f].v[v];
            float ss;
            const float r = ht_point(c, qm, qc, qp, pofs + v, omega, &ss);
            const bool in = z_in && row_in && x >= d.lo[0] && x < d.hi[0];
            outv[v] = in ? r : qc[pofs + v];
            if (in && z_own && row_own) acc += (double)ss * (double)ss;
          }
        }
        float eout = 0.f;
        if (edge) {
          float c[12];
#pragma unroll
          for (int f = 0; f < 12; f++)
            c[f] = reinterpret_cast<const float *>(cs + f * kHtField)[ecofs];
          float ss;
          const float r = ht_point(c, qm, qc, qp, epofs, omega, &ss);
          const bool in = z_in && ey >= d.lo[1] && ey < d.hi[1] && ex >= d.lo[0] && ex < d.hi[0];
          eout = in ? r : qc[epofs];
        }
        ht_release(&e1[pm.slot], lane);  // input plane z-1 is done
        ht_release(&ec[pc.slot], lane);  // the second sweep holds its own claim
        ring_next(pc, kHtSC);
        // The first-sweep plane z into the next stage of R2.
        if (p2.round > 0 && !ht_wait(&e2[p2.slot], (p2.round - 1) & 1)) {
          bad = true;
          break;
        }
        float *dst = reinterpret_cast<float *>(r2 + p2.slot * kHtStage2);
        *reinterpret_cast<float4 *>(dst + cofs) = make_float4(outv[0], outv[1], outv[2], outv[3]);
        if (edge) dst[ecofs] = eout;
        ht_release(&f2[p2.slot], lane);
        ring_next(p2, kHtS2);
        pm = pz;
        pz = pp;
      }
      if (bad) break;
      // The last two input planes were never a plane z-1.
      ht_release(&e1[pm.slot], lane);
      ht_release(&e1[pz.slot], lane);
      p1 = pz;
      ring_next(p1, kHtS1);
    }
  } else {
    // ---- stage 2: the second sweep of the tile from R2 and the coefficient
    // stages of the output planes; thread t owns 4 x points of tile row t/16.
    const int t = tid - 32 - 32 * kHtW1;
    const int tx = t % (kHtTX / kHtV), row = t / (kHtTX / kHtV);
    const int ofs = (row + 1) * kHtBX + 4 + tx * kHtV;
    RingPos p2{0, 0}, pc{0, 0};
    for (int64_t item = blockIdx.x; item < hg.items && !bad; item += gridDim.x) {
      int x0, y0, zb, nzl;
      item_geom(item, x0, y0, zb, nzl);
      const int xg = x0 + tx * kHtV, yg = y0 + row;
      const bool row_in = yg >= d.lo[1] && yg < d.hi[1];
      const bool xvec = xg >= d.lo[0] && xg + kHtV <= d.hi[0];
      // Coefficient plane zb-1 (the first sweep's halo plane) is not read here.
      if (!ht_wait(&fc[pc.slot], pc.round & 1)) {
        bad = true;
        break;
      }
      ht_release(&ec[pc.slot], lane);
      ring_next(pc, kHtSC);
      RingPos pm = p2, pz = p2;
      ring_next(pz, kHtS2);
      RingPos pp = pz;
      bad = !ht_wait(&f2[pm.slot], pm.round & 1) || !ht_wait(&f2[pz.slot], pz.round & 1);
      int64_t off = (int64_t)xg + (int64_t)yg * sy + (int64_t)zb * sz;
      for (int i = 0; i < nzl && !bad; i++) {
        ring_next(pp, kHtS2);
        if (!ht_wait(&f2[pp.slot], pp.round & 1) || !ht_wait(&fc[pc.slot], pc.round & 1)) {
          bad = true;
          break;
        }
        const float *qm = reinterpret_cast<const float *>(r2 + pm.slot * kHtStage2);
        const float *qc = reinterpret_cast<const float *>(r2 + pz.slot * kHtStage2);
        const float *qp = reinterpret_cast<const float *>(r2 + pp.slot * kHtStage2);
        const unsigned char *cs = rc + pc.slot * kHtStageC;
        if (row_in) {
          Vec16<float> co[12];
#pragma unroll
          for (int f = 0; f < 12; f++)
            co[f] = lds16(reinterpret_cast<const float *>(cs + f * kHtField) + ofs);
          float outv[kHtV];
#pragma unroll
          for (int v = 0; v < kHtV; v++) {
            float c[12];
#pragma unroll
            for (int f = 0; f < 12; f++) c[f] = co[f].v[v];
            float ss;
            outv[v] = ht_point(c, qm, qc, qp, ofs + v, omega, &ss);
            if (xg + v >= d.lo[0] && xg + v < d.hi[0]) acc += (double)ss * (double)ss;
          }
          float *dst = pout + off;
          if (xvec) {
            *reinterpret_cast<float4 *>(dst) = make_float4(outv[0], outv[1], outv[2], outv[3]);
          } else {
#pragma unroll
            for (int v = 0; v < kHtV; v++)
              if (xg + v >= d.lo[0] && xg + v < d.hi[0]) dst[v] = outv[v];
          }
        }
        ht_release(&ec[pc.slot], lane);
        ring_next(pc, kHtSC);
        ht_release(&e2[pm.slot], lane);
        pm = pz;
        pz = pp;
        off += sz;
      }
      if (bad) break;
      // Coefficient plane zb+nzl (the first sweep's far halo plane).
      if (!ht_wait(&fc[pc.slot], pc.round & 1)) {
        bad = true;
        break;
      }
      ht_release(&ec[pc.slot], lane);
      ring_next(pc, kHtSC);
      ht_release(&e2[pm.slot], lane);
      ht_release(&e2[pz.slot], lane);
      p2 = pz;
      ring_next(p2, kHtS2);
    }
  }

  // ---- residuals: per sweep one partial per CTA (fixed order), the last
  // CTA adds all partials in index order into the sweep's map history. All
  // consumer warps arrive here, a timed-out one too.
  constexpr int nct = 32 * (kHtW1 + kHtW2);
  const int cw = warp - 1;  // consumer warp 0..8
  if (bad && lane == 0) atomicExch(&flags[1], 1);
  if (bad && lane == 0) atomicExch(err, 1);
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
  // Warps 0..4 of the consumers sum sweep 1, warps 5..8 sweep 2.
  const bool first = cw < kHtW1;
  const Residual &R = first ? res1 : res2;
  const int tg = first ? tid - 32 : tid - 32 - 32 * kHtW1;
  const int ng = first ? 32 * kHtW1 : 32 * kHtW2;
  double s = 0.0;
  for (unsigned i = tg; i < gridDim.x; i += ng) s += __ldcg(&R.partials[i]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  consumer_bar(nct);
  if (lane == 0) scratch[cw] = s;
  consumer_bar(nct);
  if (tid == 32 || tid == 32 + 32 * kHtW1) {
    double sum = 0.0;
    const int w0 = first ? 0 : kHtW1, w1 = first ? kHtW1 : kHtW1 + kHtW2;
    for (int w = w0; w < w1; w++) sum += scratch[w];
    const unsigned c = *R.counter;
    R.history[c % (unsigned)R.history_len] = sum;
    *R.counter = c + 1;
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
