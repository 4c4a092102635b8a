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

// One tile of a Himeno sweep: the (TX x TY) column at (tile_x, tile_y) over
// z chunk zc. Called by every thread of the CTA; `smem` is the CTA's 128-byte
// aligned dynamic shared memory. Consumer threads add sum(ss*ss) of their
// points to *acc (FP64). Returns true in threads that must take part in a
// following consumer barrier (the consumer threads), false in the producer
// warp. A timeout sets *bad_out.
__device__ __forceinline__ bool himeno_tile(const CUtensorMap *tin, float *pout,
                                            const HimenoCoef cf, int64_t sy, int64_t sz,
                                            const Dom3 d, float omega, const HimenoGeom geo,
                                            int tile_x, int tile_y, int zc, int *err,
                                            unsigned char *smem, double *acc_out,
                                            bool *bad_out) {
  constexpr int V = 4;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *empty = full + 32;
  unsigned char *ring = smem + 768;

  const int S = geo.stages;
  const int nct = geo.tx_threads * geo.ty_threads;
  const int ncw = nct >> 5;
  const int TX = geo.tx_threads * V, TY = geo.ty_threads;
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
    mbar_fence_init();
  }
  __syncthreads();

  if (tid >= nct) {
    if (tid != nct) return false;
    tma_prefetch_desc(tin);
    const uint32_t bytes = (uint32_t)(geo.bx * geo.by * sizeof(float));
    int slot = 0, round = 0, issued = 0;
    bool ok = true;
    for (int j = 0; j < np; j++) {
      if (round > 0 && !mbar_wait_bounded(&empty[slot], (round - 1) & 1)) {
        ok = false;
        break;
      }
      mbar_arrive_expect_tx(&full[slot], bytes);
      tma_load_3d(ring + slot * geo.stage_bytes, tin, &full[slot], x0 - V + geo.ax0,
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
    return false;
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
  if (bad && lane == 0) atomicExch(err, 1);
  *acc_out += acc;
  *bad_out = bad;
  return true;
}

}  // namespace psb
