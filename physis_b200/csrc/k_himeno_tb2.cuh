// Himeno two-sweep tile machinery (temporal blocking of depth 2), shared by
// the single-grid pass (k_himeno_tb2.cu) and the batched kernel (batch.cu).
//
// One tile of TX x TY points over a z chunk advances two sweeps. Rings
// (all in one CTA's shared memory, positions carried from tile to tile):
//  R1  input pressure planes, box TX+8 x TY+4 (the tile with a 2-cell halo,
//      x from x0-4 so the box starts on 16 bytes); one producer arrival,
//      one release per stage-1 warp;
//  RC  the twelve coefficient boxes of a plane, TX+8 x TY+2 (a 1-cell
//      halo), field f at f * kHtField; one producer arrival, one release
//      per stage-1 and per stage-2 warp;
//  R2  first-sweep planes over the tile and its 1-cell halo, laid out like
//      one coefficient box; one arrival per stage-1 warp, one release per
//      stage-2 warp.
// Stage 1 (5 warps) computes the first sweep over (TX+2) x (TY+2) points
// per plane (64-point rows as float4 vectors, the two halo columns as 20
// scalar points); points outside the domain keep the input value, as a
// sweep that never writes them would. Stage 2 (4 warps) computes the second
// sweep of the tile from R2 and stores it, or (copy) stores the first sweep
// itself, which makes a one-sweep pass of the same rings. Both use the
// single-sweep arithmetic (himeno_point), so results equal single sweeps
// bit for bit.
#pragma once

#include "k_himeno.cuh"

namespace psb {

constexpr int kHtTX = 64, kHtTY = 8, kHtV = 4;
constexpr int kHtBX = kHtTX + 8;           // every box: x from x0 - 4
constexpr int kHtBY1 = kHtTY + 4;          // input p: y from y0 - 2
constexpr int kHtBY2 = kHtTY + 2;          // first sweep and coefficients: y from y0 - 1
// Ring depths (stages) of R1, R2 and RC; build options for measurement.
#ifndef PSB_HT_S1
#define PSB_HT_S1 6
#endif
#ifndef PSB_HT_S2
#define PSB_HT_S2 4
#endif
#ifndef PSB_HT_SC
#define PSB_HT_SC 4
#endif
constexpr int kHtS1 = PSB_HT_S1, kHtS2 = PSB_HT_S2, kHtSC = PSB_HT_SC;
static_assert(kHtS1 <= 8 && kHtS2 <= 8 && kHtSC <= 8, "eight barrier slots per ring");
constexpr int kHtStage1 = (kHtBX * kHtBY1 * 4 + 127) / 128 * 128;
constexpr int kHtStage2 = (kHtBX * kHtBY2 * 4 + 127) / 128 * 128;
constexpr int kHtField = kHtStage2;        // one coefficient box
constexpr int kHtStageC = 12 * kHtField;
constexpr int kHtW1 = 5, kHtW2 = 4;        // stage-1 and stage-2 warps
constexpr int kHtRingBytes = kHtS1 * kHtStage1 + kHtS2 * kHtStage2 + kHtSC * kHtStageC;
static_assert(kHtTX / kHtV * (kHtTY + 2) == 32 * kHtW1, "stage-1 threads cover the halo rows");
static_assert(kHtTX / kHtV * kHtTY == 32 * kHtW2, "stage-2 threads cover the tile");

struct HtRings {
  uint64_t *f1, *e1, *f2, *e2, *fc, *ec;  // full/empty barriers (8 slots each)
  unsigned char *r1, *r2, *rc;
};

// Barriers at bars[0..48) and rings from `rings` (kHtRingBytes).
__device__ __forceinline__ HtRings ht_rings(uint64_t *bars, unsigned char *rings) {
  HtRings R;
  R.f1 = bars;
  R.e1 = bars + 8;
  R.f2 = bars + 16;
  R.e2 = bars + 24;
  R.fc = bars + 32;
  R.ec = bars + 40;
  R.r1 = rings;
  R.r2 = R.r1 + kHtS1 * kHtStage1;
  R.rc = R.r2 + kHtS2 * kHtStage2;
  return R;
}

__device__ __forceinline__ void ht_init(const HtRings &R) {
  for (int i = 0; i < kHtS1; i++) {
    mbar_init(&R.f1[i], 1);
    mbar_init(&R.e1[i], kHtW1);
  }
  for (int i = 0; i < kHtS2; i++) {
    mbar_init(&R.f2[i], kHtW1);
    mbar_init(&R.e2[i], kHtW2);
  }
  for (int i = 0; i < kHtSC; i++) {
    mbar_init(&R.fc[i], 1);
    mbar_init(&R.ec[i], kHtW1 + kHtW2);
  }
}

// 19 pressure values around offset o of three planes with row length kHtBX
// (m: z-1, c: z, p: z+1) and the point's 12 coefficients.
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

// Producer (one thread): input planes zb-2 .. zb+nzl+1 into R1 and
// coefficient planes zb-1 .. zb+nzl into RC, each RC plane issued after the
// R1 plane the first sweep needs with it, so neither ring waits on a stage
// of the other that is not yet issued. coef: 12 tensor maps, one per field.
// (ax0, ay0, az0): tensor coordinates of logical (0,0,0). False if a
// bounded wait gave up.
__device__ __forceinline__ bool ht_produce_tile(const HtRings &R, RingPos &p1, RingPos &pc,
                                                const CUtensorMap *tin, const CUtensorMap *coef,
                                                int ax0, int ay0, int az0, int x0, int y0,
                                                int zb, int nzl) {
  auto put1 = [&](int z) -> bool {
    if (p1.round > 0 && !mbar_wait_bounded(&R.e1[p1.slot], (p1.round - 1) & 1)) return false;
    mbar_arrive_expect_tx(&R.f1[p1.slot], (uint32_t)(kHtBX * kHtBY1 * 4));
    tma_load_3d(R.r1 + p1.slot * kHtStage1, tin, &R.f1[p1.slot], x0 - 4 + ax0, y0 - 2 + ay0,
                z + az0);
    ring_next(p1, kHtS1);
    return true;
  };
  auto putc = [&](int z) -> bool {
    if (pc.round > 0 && !mbar_wait_bounded(&R.ec[pc.slot], (pc.round - 1) & 1)) return false;
    mbar_arrive_expect_tx(&R.fc[pc.slot], (uint32_t)(12 * kHtBX * kHtBY2 * 4));
    unsigned char *dst = R.rc + pc.slot * kHtStageC;
    for (int f = 0; f < 12; f++)
      tma_load_3d(dst + f * kHtField, coef + f, &R.fc[pc.slot], x0 - 4 + ax0, y0 - 1 + ay0,
                  z + az0);
    ring_next(pc, kHtSC);
    return true;
  };
  if (!put1(zb - 2) || !put1(zb - 1)) return false;
  for (int j = 0; j < nzl + 2; j++)
    if (!put1(zb + j) || !putc(zb - 1 + j)) return false;
  return true;
}

// After a producer gave up: wait (bounded) for its copies in flight.
__device__ __forceinline__ void ht_drain(const HtRings &R, RingPos p1, RingPos pc) {
  ring_drain(Ring{R.f1, R.e1, R.r1, kHtS1, kHtStage1}, p1);
  ring_drain(Ring{R.fc, R.ec, R.rc, kHtSC, kHtStageC}, pc);
}

// Stage-1 warps (thread t in [0, 160)): the first sweep of one tile into R2.
// Thread t owns 4 x points of halo row t / 16 (y = y0 - 1 + row); every
// eighth thread also owns one of the 20 edge points (x0 - 1 and x0 + TX of
// each row). With acc_on, the FP64 sum of ss*ss over the tile's own domain
// points is added to *acc. False (warp-uniformly) if a bounded wait gave up.
__device__ __forceinline__ bool ht_stage1_tile(const HtRings &R, RingPos &p1, RingPos &pc,
                                               RingPos &p2, int t, int lane, const Dom3 d,
                                               float omega, int x0, int y0, int zb, int nzl,
                                               bool acc_on, double *acc) {
  const int tx = t % (kHtTX / kHtV), row = t / (kHtTX / kHtV);
  const int cofs = row * kHtBX + 4 + tx * kHtV;        // R2 / RC offset of the vector
  const int pofs = (row + 1) * kHtBX + 4 + tx * kHtV;  // R1 offset of the vector
  const bool edge = (t & 7) == 0;
  const int e = t >> 3;                                // 0..19
  const int ecol = e / (kHtTY + 2), erow = e % (kHtTY + 2);
  const int ex_off = ecol ? 4 + kHtTX : 3;
  const int ecofs = erow * kHtBX + ex_off, epofs = (erow + 1) * kHtBX + ex_off;
  const int xg = x0 + tx * kHtV, yg = y0 - 1 + row;
  const int ex = ecol ? x0 + kHtTX : x0 - 1, ey = y0 - 1 + erow;
  const bool row_in = yg >= d.lo[1] && yg < d.hi[1];
  const bool row_own = row_in && row >= 1 && row <= kHtTY;
  RingPos pm = p1, pz = p1;  // input planes z-1 and z
  ring_next(pz, kHtS1);
  RingPos pp = pz;
  if (!ht_wait(&R.f1[pm.slot], pm.round & 1) || !ht_wait(&R.f1[pz.slot], pz.round & 1))
    return false;
  double a = 0.0;
  for (int j = 0; j < nzl + 2; j++) {
    const int z = zb - 1 + j;
    ring_next(pp, kHtS1);
    if (!ht_wait(&R.f1[pp.slot], pp.round & 1) || !ht_wait(&R.fc[pc.slot], pc.round & 1))
      return false;
    const float *qm = reinterpret_cast<const float *>(R.r1 + pm.slot * kHtStage1);
    const float *qc = reinterpret_cast<const float *>(R.r1 + pz.slot * kHtStage1);
    const float *qp = reinterpret_cast<const float *>(R.r1 + pp.slot * kHtStage1);
    const unsigned char *cs = R.rc + pc.slot * kHtStageC;
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
        if (acc_on && in && z_own && row_own) a += (double)ss * (double)ss;
      }
    }
    float eout = 0.f;
    if (edge) {
      float c[12];
#pragma unroll
      for (int f = 0; f < 12; f++) c[f] = reinterpret_cast<const float *>(cs + f * kHtField)[ecofs];
      float ss;
      const float r = ht_point(c, qm, qc, qp, epofs, omega, &ss);
      const bool in = z_in && ey >= d.lo[1] && ey < d.hi[1] && ex >= d.lo[0] && ex < d.hi[0];
      eout = in ? r : qc[epofs];
    }
    ht_release(&R.e1[pm.slot], lane);  // input plane z-1 is done
    ht_release(&R.ec[pc.slot], lane);  // stage 2 holds its own claim on the stage
    ring_next(pc, kHtSC);
    // The first-sweep plane z into the next stage of R2.
    if (p2.round > 0 && !ht_wait(&R.e2[p2.slot], (p2.round - 1) & 1)) return false;
    float *dst = reinterpret_cast<float *>(R.r2 + p2.slot * kHtStage2);
    *reinterpret_cast<float4 *>(dst + cofs) = make_float4(outv[0], outv[1], outv[2], outv[3]);
    if (edge) dst[ecofs] = eout;
    ht_release(&R.f2[p2.slot], lane);
    ring_next(p2, kHtS2);
    pm = pz;
    pz = pp;
  }
  // The last two input planes were never a plane z-1.
  ht_release(&R.e1[pm.slot], lane);
  ht_release(&R.e1[pz.slot], lane);
  p1 = pz;
  ring_next(p1, kHtS1);
  *acc += a;
  return true;
}

// Stage-2 warps (thread t in [0, 128)): the second sweep of the tile from R2
// and the coefficient stages of its planes, stored to pout (copy: the first
// sweep itself is stored). Thread t owns 4 x points of tile row t / 16.
// With acc_on (and not copy), the FP64 sum of ss*ss over the tile's domain
// points is added to *acc. False (warp-uniformly) if a bounded wait gave up.
__device__ __forceinline__ bool ht_stage2_tile(const HtRings &R, RingPos &p2, RingPos &pc, int t,
                                               int lane, float *pout, int64_t sy, int64_t sz,
                                               const Dom3 d, float omega, int x0, int y0,
                                               int zb, int nzl, bool copy, bool acc_on,
                                               double *acc) {
  const int tx = t % (kHtTX / kHtV), row = t / (kHtTX / kHtV);
  const int ofs = (row + 1) * kHtBX + 4 + tx * kHtV;
  const int xg = x0 + tx * kHtV, yg = y0 + row;
  const bool row_in = yg >= d.lo[1] && yg < d.hi[1];
  const bool xvec = xg >= d.lo[0] && xg + kHtV <= d.hi[0];
  // Coefficient plane zb-1 (the first sweep's near halo plane) is not read.
  if (!ht_wait(&R.fc[pc.slot], pc.round & 1)) return false;
  ht_release(&R.ec[pc.slot], lane);
  ring_next(pc, kHtSC);
  RingPos pm = p2, pz = p2;
  ring_next(pz, kHtS2);
  RingPos pp = pz;
  if (!ht_wait(&R.f2[pm.slot], pm.round & 1) || !ht_wait(&R.f2[pz.slot], pz.round & 1))
    return false;
  double a = 0.0;
  int64_t off = (int64_t)xg + (int64_t)yg * sy + (int64_t)zb * sz;
  for (int i = 0; i < nzl; i++) {
    ring_next(pp, kHtS2);
    if (!ht_wait(&R.f2[pp.slot], pp.round & 1) || !ht_wait(&R.fc[pc.slot], pc.round & 1))
      return false;
    const float *qm = reinterpret_cast<const float *>(R.r2 + pm.slot * kHtStage2);
    const float *qc = reinterpret_cast<const float *>(R.r2 + pz.slot * kHtStage2);
    const float *qp = reinterpret_cast<const float *>(R.r2 + pp.slot * kHtStage2);
    const unsigned char *cs = R.rc + pc.slot * kHtStageC;
    if (row_in) {
      float outv[kHtV];
      if (copy) {
#pragma unroll
        for (int v = 0; v < kHtV; v++) outv[v] = qc[ofs + v];
      } else {
        Vec16<float> co[12];
#pragma unroll
        for (int f = 0; f < 12; f++)
          co[f] = lds16(reinterpret_cast<const float *>(cs + f * kHtField) + ofs);
#pragma unroll
        for (int v = 0; v < kHtV; v++) {
          float c[12];
#pragma unroll
          for (int f = 0; f < 12; f++) c[f] = co[f].v[v];
          float ss;
          outv[v] = ht_point(c, qm, qc, qp, ofs + v, omega, &ss);
          if (acc_on && xg + v >= d.lo[0] && xg + v < d.hi[0]) a += (double)ss * (double)ss;
        }
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
    ht_release(&R.ec[pc.slot], lane);
    ring_next(pc, kHtSC);
    ht_release(&R.e2[pm.slot], lane);
    pm = pz;
    pz = pp;
    off += sz;
  }
  // Coefficient plane zb+nzl (the first sweep's far halo plane).
  if (!ht_wait(&R.fc[pc.slot], pc.round & 1)) return false;
  ht_release(&R.ec[pc.slot], lane);
  ring_next(pc, kHtSC);
  ht_release(&R.e2[pm.slot], lane);
  ht_release(&R.e2[pz.slot], lane);
  p2 = pz;
  ring_next(p2, kHtS2);
  *acc += a;
  return true;
}

}  // namespace psb
