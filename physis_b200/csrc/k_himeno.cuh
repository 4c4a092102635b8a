// Himeno tile machinery shared by the single-grid kernels (k_himeno.cu) and
// the batched persistent kernels (batch.cu).
#pragma once

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

// Consumer warps, one tile of a Himeno sweep: planes zb-1 .. zb+nzl of p
// around the (TX x TY) column at (x0, y0), from ring position p on (advanced
// past all nzl + 2 planes, every one released). The twelve coefficient
// fields are streamed from global memory with 16-byte loads issued before
// the plane wait. Each consumer thread adds sum(ss*ss) of its points to *acc
// (FP64). `coef(i)` gives the origin of coefficient field i; callers pass a
// function that reads it where it is cheapest (a kernel parameter, or shared
// memory, so 12 pointers need not occupy registers). Returns false
// (warp-uniformly) if a bounded wait gave up.
template <typename CoefFn>
__device__ __forceinline__ bool himeno_consume(const Ring &R, RingPos &p, float *pout,
                                               CoefFn coef, int64_t sy, int64_t sz,
                                               const Dom3 d, float omega, const HimenoGeom geo,
                                               int x0, int y0, int zb, int nzl, double *acc_out) {
  constexpr int V = 4;
  const int S = R.S;
  const int tid = threadIdx.x;
  const int tx = tid % geo.tx_threads, ty = tid / geo.tx_threads;
  const int lane = tid & 31;
  const int BX = geo.bx;
  const int rc = (ty + 1) * BX + V + tx * V;
  const int xg0 = x0 + tx * V;
  const int yg = y0 + ty;
  const bool row_in = yg >= d.lo[1] && yg < d.hi[1];
  const bool vec_ok = xg0 + V <= geo.nx;
  const bool xvec = xg0 >= d.lo[0] && xg0 + V <= d.hi[0];
  auto wait_plane = [&](const RingPos &q) -> bool {
    bool ok = mbar_wait_bounded(&R.full[q.slot], q.round & 1);
    return __all_sync(0xffffffffu, ok);
  };
  auto release = [&](int slot) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&R.empty[slot]);
  };
  auto plane_ptr = [&](int slot) -> const float * {
    return reinterpret_cast<const float *>(R.base + slot * R.stage_bytes);
  };
  double acc = 0.0;
  RingPos pm = p;  // plane z-1
  RingPos pc = p;  // plane z
  ring_next(pc, S);
  RingPos pp = pc;  // plane z+1 (advanced before use)
  bool bad = !wait_plane(pm);
  bad = bad || !wait_plane(pc);
  int64_t off = (int64_t)xg0 + (int64_t)yg * sy + (int64_t)zb * sz;
  for (int jj = 0; jj < nzl && !bad; jj++) {
    float co[12][V];
    if (row_in) {
#pragma unroll
      for (int i = 0; i < 12; i++) {
        const float *f = coef(i);
        if (vec_ok) {
          Vec16<float> q = ldg16_stream(f + off);
#pragma unroll
          for (int v = 0; v < V; v++) co[i][v] = q.v[v];
        } else {
#pragma unroll
          for (int v = 0; v < V; v++) co[i][v] = xg0 + v < geo.nx ? f[off + v] : 0.f;
        }
      }
    }
    ring_next(pp, S);
    if (!wait_plane(pp)) {
      bad = true;
      break;
    }
    const float *qm = plane_ptr(pm.slot), *qc = plane_ptr(pc.slot), *qp = plane_ptr(pp.slot);
    if (row_in) {
      float outv[V];
#pragma unroll
      for (int v = 0; v < V; v++) {
        const int o = rc + v;
        float c[12];
#pragma unroll
        for (int i = 0; i < 12; i++) c[i] = co[i][v];
        float ss;
        outv[v] = himeno_point(c, qc[o], qc[o + 1], qc[o - 1], qc[o + BX], qc[o - BX], qp[o],
                               qm[o], qp[o + BX], qp[o - BX], qm[o + BX], qm[o - BX],
                               qc[o + 1 + BX], qc[o + 1 - BX], qc[o - 1 + BX], qc[o - 1 - BX],
                               qp[o + 1], qm[o + 1], qp[o - 1], qm[o - 1], omega, &ss);
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
    release(pm.slot);
    pm = pc;
    pc = pp;
    off += sz;
  }
  *acc_out += acc;
  if (bad) return false;
  // The last two planes (z and z+1 of the last output plane).
  release(pm.slot);
  release(pc.slot);
  p = pc;
  ring_next(p, S);
  return true;
}

// Coefficient tiles of output plane z (tensor coordinates) into the next
// stage of ring RC: twelve TMA loads (maps tcoef[f * stride], boxes of
// box_bytes) completing on one barrier, field f at f * field_bytes.
__device__ __forceinline__ bool coef_produce(const Ring &RC, RingPos &p, const CUtensorMap *tcoef,
                                             int stride, int field_bytes, int box_bytes, int cx,
                                             int cy, int cz) {
  if (p.round > 0 && !mbar_wait_bounded(&RC.empty[p.slot], (p.round - 1) & 1)) return false;
  mbar_arrive_expect_tx(&RC.full[p.slot], (uint32_t)(12 * box_bytes));
  unsigned char *dst = RC.base + p.slot * RC.stage_bytes;
  for (int f = 0; f < 12; f++)
    tma_load_3d(dst + f * field_bytes, tcoef + f * stride, &RC.full[p.slot], cx, cy, cz);
  ring_next(p, RC.S);
  return true;
}

// Consumer warps, one Himeno tile with staged coefficients: planes zb-1 ..
// zb+nzl of p through ring R (as himeno_consume), and for each output plane
// one stage of ring RC holding its twelve coefficient tiles (rows of TX
// floats). Both rings are advanced past the tile, every stage released.
__device__ __forceinline__ bool himeno_consume_staged(const Ring &R, RingPos &p, const Ring &RC,
                                                      RingPos &pcoef, int tile_bytes, float *pout,
                                                      int64_t sy,
                                                      int64_t sz, const Dom3 d, float omega,
                                                      const HimenoGeom geo, int x0, int y0,
                                                      int zb, int nzl, double *acc_out) {
  constexpr int V = 4;
  const int S = R.S;
  const int tid = threadIdx.x;
  // Threads past tx_threads * ty_threads (shapes that do not divide the
  // consumer count) take part in every wait and release but own no points.
  const int tx = tid % geo.tx_threads;
  const bool active = tid / geo.tx_threads < geo.ty_threads;
  const int ty = active ? tid / geo.tx_threads : geo.ty_threads - 1;
  const int lane = tid & 31;
  const int BX = geo.bx;
  const int rc = (ty + 1) * BX + V + tx * V;
  const int co_off = (ty * geo.tx_threads * V + tx * V) * 4;  // bytes into a coefficient tile
  const int xg0 = x0 + tx * V;
  const int yg = y0 + ty;
  const bool row_in = active && yg >= d.lo[1] && yg < d.hi[1];
  const bool xvec = xg0 >= d.lo[0] && xg0 + V <= d.hi[0];
  auto wait_stage = [&](const Ring &Q, const RingPos &q) -> bool {
    bool ok = mbar_wait_bounded(&Q.full[q.slot], q.round & 1);
    return __all_sync(0xffffffffu, ok);
  };
  auto release = [&](const Ring &Q, int slot) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&Q.empty[slot]);
  };
  auto plane_ptr = [&](int slot) -> const float * {
    return reinterpret_cast<const float *>(R.base + slot * R.stage_bytes);
  };
  double acc = 0.0;
  RingPos pm = p;  // plane z-1
  RingPos pc = p;  // plane z
  ring_next(pc, S);
  RingPos pp = pc;  // plane z+1 (advanced before use)
  bool bad = !wait_stage(R, pm);
  bad = bad || !wait_stage(R, pc);
  int64_t off = (int64_t)xg0 + (int64_t)yg * sy + (int64_t)zb * sz;
  for (int jj = 0; jj < nzl && !bad; jj++) {
    ring_next(pp, S);
    if (!wait_stage(R, pp) || !wait_stage(RC, pcoef)) {
      bad = true;
      break;
    }
    const float *qm = plane_ptr(pm.slot), *qc = plane_ptr(pc.slot), *qp = plane_ptr(pp.slot);
    if (row_in) {
      const unsigned char *cs = RC.base + pcoef.slot * RC.stage_bytes + co_off;
      Vec16<float> co[12];
#pragma unroll
      for (int i = 0; i < 12; i++)
        co[i] = lds16(reinterpret_cast<const float *>(cs + i * tile_bytes));
      float outv[V];
#pragma unroll
      for (int v = 0; v < V; v++) {
        const int o = rc + v;
        float c[12];
#pragma unroll
        for (int i = 0; i < 12; i++) c[i] = co[i].v[v];
        float ss;
        outv[v] = himeno_point(c, qc[o], qc[o + 1], qc[o - 1], qc[o + BX], qc[o - BX], qp[o],
                               qm[o], qp[o + BX], qp[o - BX], qm[o + BX], qm[o - BX],
                               qc[o + 1 + BX], qc[o + 1 - BX], qc[o - 1 + BX], qc[o - 1 - BX],
                               qp[o + 1], qm[o + 1], qp[o - 1], qm[o - 1], omega, &ss);
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
    release(RC, pcoef.slot);
    ring_next(pcoef, RC.S);
    release(R, pm.slot);  // plane z-1 is done for this warp
    pm = pc;
    pc = pp;
    off += sz;
  }
  *acc_out += acc;
  if (bad) return false;
  release(R, pm.slot);
  release(R, pc.slot);
  p = pc;
  ring_next(p, S);
  return true;
}

// One tile of a Himeno sweep as a whole CTA (single-grid kernels): the
// (TX x TY) column at (tile_x, tile_y) over z chunk zc. `smem` is the CTA's
// 128-byte aligned dynamic shared memory. Consumer threads add sum(ss*ss) of
// their points to *acc (FP64). Returns true in threads that must take part
// in a following consumer barrier (the consumer threads), false in the
// producer warp. A timeout sets *bad_out.
__device__ __forceinline__ bool himeno_tile(const CUtensorMap *tin, float *pout,
                                            const HimenoCoef cf, int64_t sy, int64_t sz,
                                            const Dom3 d, float omega, const HimenoGeom geo,
                                            int tile_x, int tile_y, int zc, int *err,
                                            unsigned char *smem, double *acc_out,
                                            bool *bad_out) {
  constexpr int V = 4;
  const Ring R{reinterpret_cast<uint64_t *>(smem), reinterpret_cast<uint64_t *>(smem) + 32,
               smem + 768, geo.stages, geo.stage_bytes};
  const int nct = geo.tx_threads * geo.ty_threads;
  const int TX = geo.tx_threads * V, TY = geo.ty_threads;
  const int x0 = geo.x_base + tile_x * TX;
  const int y0 = d.lo[1] + tile_y * TY;
  const int zb = d.lo[2] + zc * geo.zchunk;
  const int nzl = min(zb + geo.zchunk, d.hi[2]) - zb;
  const int tid = threadIdx.x;

  if (tid == 0) ring_init(R, nct >> 5);
  __syncthreads();

  RingPos pos{0, 0};
  if (tid >= nct) {
    if (tid != nct) return false;
    tma_prefetch_desc(tin);
    const uint32_t bytes = (uint32_t)(geo.bx * geo.by * sizeof(float));
    if (!ring_produce(R, pos, tin, bytes, x0 - V + geo.ax0, y0 - 1 + geo.ay0, zb - 1 + geo.az0,
                      nzl + 2)) {
      atomicExch(err, 1);
      ring_drain(R, pos);
    }
    return false;
  }
  const bool ok = himeno_consume(R, pos, pout, [&](int i) { return cf.f[i]; }, sy, sz, d, omega,
                                 geo, x0, y0, zb, nzl, acc_out);
  if (!ok && (tid & 31) == 0) atomicExch(err, 1);
  *bad_out = !ok;
  return true;
}

}  // namespace psb
