// 7-point diffusion tile machinery shared by the single-grid kernels
// (k_diffusion7.cu) and the batched persistent kernels (batch.cu).
#pragma once

#include "device.cuh"

namespace psb {

template <typename T>
struct C7 {
  T ce, cw, cn, cs, ct, cb, cc;
};

// FAST = false: the reference's roundings (every product and sum rounded).
// FAST = true: the contracted form of the same term order -- the first
// product rounded, then each further term added by one fused multiply-add
// (one rounding per term instead of two). It is no longer bit-identical to
// the reference CPU target; on the C2 field and on random inputs in [0, 1)
// one step differs from it by at most 4 ulp, and its error against an FP64
// evaluation is no larger than the exact form's.
__device__ __forceinline__ float xfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double xfma(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T, bool FAST = false>
__device__ __forceinline__ T diff7_point(const C7<T> &k, T c, T w, T e, T n, T s, T b, T t) {
  T v = xmul(k.cc, c);
  if constexpr (FAST) {
    v = xfma(k.cw, w, v);
    v = xfma(k.ce, e, v);
    v = xfma(k.cs, s, v);
    v = xfma(k.cn, n, v);
    v = xfma(k.cb, b, v);
    v = xfma(k.ct, t, v);
  } else {
    v = xadd(v, xmul(k.cw, w));
    v = xadd(v, xmul(k.ce, e));
    v = xadd(v, xmul(k.cs, s));
    v = xadd(v, xmul(k.cn, n));
    v = xadd(v, xmul(k.cb, b));
    v = xadd(v, xmul(k.ct, t));
  }
  return v;
}

// Four (float) or two (double) consecutive x points of one row. c/n/s/b/t
// are the 16-byte vectors of the points' own column in the planes/rows
// around them; wl/er are the scalars left and right of the vector. The w
// and e neighbours of a point are its vector's own elements shifted by one,
// so the products cw*w and ce*e come from cw*c and ce*c of the neighbouring
// lanes plus one scalar product each at the ends. The float form computes
// products of natural element pairs with the packed sm_100 f32x2 multiply
// (every lane an IEEE round-to-nearest product) and sums them with scalar
// round-to-nearest adds in the reference order. The adds stay scalar on
// purpose: a packed add that consumes a packed product is fused into a
// packed FMA by the compiler even when both carry an explicit .rn, which
// would change the rounding; a scalar add of a packed product is not.
// xfix marks clamped x faces inside the vector: bit 4 = the first point is
// x = 0 (its w is c), bit v = point v is x = nx-1 (its e is c).
template <typename T>
struct K7 {
  C7<T> s;
};
template <>
struct K7<float> {
  C7<float> s;
  float2 ce, cw, cn, cs, ct, cb, cc;
};

template <typename T>
__device__ __forceinline__ K7<T> make_k7(const C7<T> &c) {
  K7<T> k;
  k.s = c;
  if constexpr (sizeof(T) == 4) {
    k.ce = make_float2(c.ce, c.ce);
    k.cw = make_float2(c.cw, c.cw);
    k.cn = make_float2(c.cn, c.cn);
    k.cs = make_float2(c.cs, c.cs);
    k.ct = make_float2(c.ct, c.ct);
    k.cb = make_float2(c.cb, c.cb);
    k.cc = make_float2(c.cc, c.cc);
  }
  return k;
}

__device__ __forceinline__ void mul4(float2 k, const Vec16<float> &x, float *p) {
  const float2 lo = __fmul2_rn(k, make_float2(x.v[0], x.v[1]));
  const float2 hi = __fmul2_rn(k, make_float2(x.v[2], x.v[3]));
  p[0] = lo.x;
  p[1] = lo.y;
  p[2] = hi.x;
  p[3] = hi.y;
}

// Contracted row (FAST): pairs of points with the packed sm_100 f32x2
// multiply and fused multiply-add, in the term order of diff7_point<FAST>;
// the w and e operands of each pair are the row's own elements shifted by
// one (wl and er at the ends), with the clamped x faces selected first.
__device__ __forceinline__ Vec16<float> diff7_row_fast(const K7<float> &k, const Vec16<float> &c,
                                                       float wl, float er, const Vec16<float> &n,
                                                       const Vec16<float> &s,
                                                       const Vec16<float> &b,
                                                       const Vec16<float> &t, unsigned xfix) {
  float w0 = wl, e0 = c.v[1], e1 = c.v[2], e2 = c.v[3], e3 = er;
  if (xfix) {
    if (xfix & 16u) w0 = c.v[0];
    if (xfix & 1u) e0 = c.v[0];
    if (xfix & 2u) e1 = c.v[1];
    if (xfix & 4u) e2 = c.v[2];
    if (xfix & 8u) e3 = c.v[3];
  }
  float2 lo = __fmul2_rn(k.cc, make_float2(c.v[0], c.v[1]));
  float2 hi = __fmul2_rn(k.cc, make_float2(c.v[2], c.v[3]));
  lo = __ffma2_rn(k.cw, make_float2(w0, c.v[0]), lo);
  hi = __ffma2_rn(k.cw, make_float2(c.v[1], c.v[2]), hi);
  lo = __ffma2_rn(k.ce, make_float2(e0, e1), lo);
  hi = __ffma2_rn(k.ce, make_float2(e2, e3), hi);
  lo = __ffma2_rn(k.cs, make_float2(s.v[0], s.v[1]), lo);
  hi = __ffma2_rn(k.cs, make_float2(s.v[2], s.v[3]), hi);
  lo = __ffma2_rn(k.cn, make_float2(n.v[0], n.v[1]), lo);
  hi = __ffma2_rn(k.cn, make_float2(n.v[2], n.v[3]), hi);
  lo = __ffma2_rn(k.cb, make_float2(b.v[0], b.v[1]), lo);
  hi = __ffma2_rn(k.cb, make_float2(b.v[2], b.v[3]), hi);
  lo = __ffma2_rn(k.ct, make_float2(t.v[0], t.v[1]), lo);
  hi = __ffma2_rn(k.ct, make_float2(t.v[2], t.v[3]), hi);
  Vec16<float> r;
  r.v[0] = lo.x;
  r.v[1] = lo.y;
  r.v[2] = hi.x;
  r.v[3] = hi.y;
  return r;
}

template <typename T, bool FAST = false>
__device__ __forceinline__ Vec16<T> diff7_row(const K7<T> &k, const Vec16<T> &c, T wl, T er,
                                              const Vec16<T> &n, const Vec16<T> &s,
                                              const Vec16<T> &b, const Vec16<T> &t,
                                              unsigned xfix) {
  constexpr int V = Vec16<T>::N;
  if constexpr (FAST && sizeof(T) == 4) {
    return diff7_row_fast(k, c, wl, er, n, s, b, t, xfix);
  } else if constexpr (FAST) {
    Vec16<T> r;
#pragma unroll
    for (int v = 0; v < V; v++) {
      T w = v == 0 ? ((xfix & 16u) ? c.v[0] : wl) : c.v[v - 1];
      T e = (xfix & (1u << v)) ? c.v[v] : (v == V - 1 ? er : c.v[v + 1]);
      r.v[v] = diff7_point<T, true>(k.s, c.v[v], w, e, n.v[v], s.v[v], b.v[v], t.v[v]);
    }
    return r;
  }
  T pcc[V], pcw[V], pce[V], ps[V], pn[V], pb[V], pt[V];
  if constexpr (sizeof(T) == 4) {
    mul4(k.cc, c, pcc);
    mul4(k.cw, c, pcw);
    mul4(k.ce, c, pce);
    mul4(k.cs, s, ps);
    mul4(k.cn, n, pn);
    mul4(k.cb, b, pb);
    mul4(k.ct, t, pt);
  } else {
#pragma unroll
    for (int v = 0; v < V; v++) {
      pcc[v] = xmul(k.s.cc, c.v[v]);
      pcw[v] = xmul(k.s.cw, c.v[v]);
      pce[v] = xmul(k.s.ce, c.v[v]);
      ps[v] = xmul(k.s.cs, s.v[v]);
      pn[v] = xmul(k.s.cn, n.v[v]);
      pb[v] = xmul(k.s.cb, b.v[v]);
      pt[v] = xmul(k.s.ct, t.v[v]);
    }
  }
  T pw[V], pe[V];
  pw[0] = xmul(k.s.cw, wl);
#pragma unroll
  for (int v = 1; v < V; v++) pw[v] = pcw[v - 1];
#pragma unroll
  for (int v = 0; v < V - 1; v++) pe[v] = pce[v + 1];
  pe[V - 1] = xmul(k.s.ce, er);
  if (xfix) {
    if (xfix & 16u) pw[0] = pcw[0];
#pragma unroll
    for (int v = 0; v < V; v++)
      if (xfix & (1u << v)) pe[v] = pce[v];
  }
  Vec16<T> r;
#pragma unroll
  for (int v = 0; v < V; v++)
    r.v[v] = xadd(xadd(xadd(xadd(xadd(xadd(pcc[v], pw[v]), pe[v]), ps[v]), pn[v]), pb[v]), pt[v]);
  return r;
}

// --------------------------------------------------------------------------
// TMA z-streaming, warp-specialised
//
// One producer thread streams input planes (box (TX+2V) x (TY+2) x 1) into a
// ring of S shared-memory stages with TMA; `full[s]` completes when a plane
// has landed, `empty[s]` when every consumer warp has finished with it.
// Consumer warps never meet at a CTA-wide barrier: each waits on the plane
// it needs and releases it when done. Each consumer thread owns V
// consecutive x points (16 bytes) of VY rows; z neighbours stay in
// registers. Faces are resolved with selects only on threads/planes that
// touch a face; all other points take a select-free path.
//
// The ring position is an explicit value (Ring, RingPos in device.cuh), so
// one ring can carry the planes of many tiles back to back: the single-grid
// kernels run one tile per CTA, the batched persistent kernel streams tile
// after tile through the same ring without draining it.
// --------------------------------------------------------------------------
struct TmaGeom {
  int ax0, ay0, az0;      // tensor-map coordinates of logical (0,0,0)
  int tiles_x, tiles_y;   // tiles over the domain
  int zchunk;             // planes per CTA
  int stages;             // ring depth
  int bx, by;             // box (elements)
  int stage_bytes;        // bytes between stages (128-aligned)
  int x_base;             // x of the first tile (domain lo rounded down)
  int tx_threads;         // consumer threads along x (TX / V)
  int ty_threads;         // consumer thread rows (TY / VY)
};

constexpr int kVY = 2;

// Per-thread accumulators of a convergence measure, filled only when a
// caller asks for them: a = sum of (new - old)^2, b = sum of new^2 (FP64).
struct TileAcc {
  double a, b;
};

// Consumer warps, one tile: planes zb-1 .. zb+nzl of the (TX x TY) column
// at (x0, y0), starting at ring position p (advanced past all nzl + 2 planes,
// every one of which is released). Output rows go to `out`; with PERIODIC
// and `images`, every written face point also stores its image in the halo
// (depth 1, one per face it lies on), which keeps the resident halo current
// for the next periodic read. With ACC the convergence terms are added to
// *acc. Returns false (warp-uniformly) if a bounded wait gave up.
template <typename T, bool PERIODIC, bool ACC, bool FAST = false>
__device__ __forceinline__ bool diff7_consume(const Ring &R, RingPos &p, const GridView out,
                                              int nx, int ny, int nz, const Dom3 d,
                                              const C7<T> k, const TmaGeom geo, int x0, int y0,
                                              int zb, int nzl, int images, TileAcc *acc,
                                              int tid = -1) {
  constexpr int V = 16 / sizeof(T);
  constexpr int VY = kVY;
  const int S = R.S;
  // tid: this thread's index among the consumer threads (whole warps; the
  // threads of the CTA by default).
  if (tid < 0) tid = threadIdx.x;
  // Threads past tx_threads * ty_threads (shapes that do not divide the
  // consumer count) take part in every wait and release but own no points.
  const int tx = tid % geo.tx_threads;
  const bool active = tid / geo.tx_threads < geo.ty_threads;
  const int ty = active ? tid / geo.tx_threads : geo.ty_threads - 1;
  const int lane = tid & 31;
  const int BX = geo.bx;
  const int xg0 = x0 + tx * V;
  const int yg0 = y0 + ty * VY;
  const int rc0 = (ty * VY + 1) * BX + V + tx * V;  // smem offset of (x0, row 0)
  // Clamped x faces inside this thread's vector (see diff7_row).
  unsigned xfix = 0;
  if (!PERIODIC) {
    if (xg0 == 0) xfix |= 16u;
#pragma unroll
    for (int v = 0; v < V; v++)
      if (xg0 + v == nx - 1) xfix |= 1u << v;
  }
  bool yedge = false;
#pragma unroll
  for (int r = 0; r < VY; r++) yedge = yedge || yg0 + r == 0 || yg0 + r == ny - 1;
  yedge = !PERIODIC && yedge;
  bool row_in[VY];
#pragma unroll
  for (int r = 0; r < VY; r++) row_in[r] = active && yg0 + r >= d.lo[1] && yg0 + r < d.hi[1];
  const bool xvec = xg0 >= d.lo[0] && xg0 + V <= d.hi[0];
  // Periodic x-face images of this thread's vector: x = 0 goes to x = nx,
  // x = nx-1 to x = -1.
  const int vlast = nx - 1 - xg0;  // element of the vector at x = nx-1, if 0 <= vlast < V
  const bool img_x0 = PERIODIC && xg0 == 0 && d.lo[0] <= 0;
  const bool img_x1 = PERIODIC && vlast >= 0 && vlast < V && nx - 1 >= d.lo[0] && nx - 1 < d.hi[0];
  const K7<T> kk = make_k7(k);

  // Every lane waits (the wait gives it visibility of the TMA data); the
  // outcome is made warp-uniform so a timeout never splits a warp.
  auto wait_plane = [&](const RingPos &q) -> bool {
    bool ok = mbar_wait_bounded(&R.full[q.slot], q.round & 1);
    return __all_sync(0xffffffffu, ok);
  };
  auto release = [&](int slot) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&R.empty[slot]);
  };
  auto plane_ptr = [&](int slot) -> const T * {
    return reinterpret_cast<const T *>(R.base + slot * R.stage_bytes);
  };
  auto store_vec = [&](T *dst, const Vec16<T> &v) {
    if (xvec) {
      stg16(dst, v);
    } else {
#pragma unroll
      for (int e = 0; e < V; e++)
        if (xg0 + e >= d.lo[0] && xg0 + e < d.hi[0]) dst[e] = v.v[e];
    }
  };

  T *o = (T *)out.origin;
  T *dst0 = o + (int64_t)xg0 + (int64_t)yg0 * out.sy + (int64_t)zb * out.sz;
  RingPos pz = p;  // plane of z (after the prologue)
  ring_next(pz, S);
  RingPos pt = pz;  // plane of z+1 (advanced before use)
  int z = zb;

  // One z step: b = plane z-1 (registers), c = plane z (registers), t is
  // loaded from the plane of z+1. Returns false on a timeout.
  auto step = [&](Vec16<T>(&vb)[VY], Vec16<T>(&vc)[VY], Vec16<T>(&vt)[VY]) -> bool {
    ring_next(pt, S);
    if (!wait_plane(pt)) return false;
    const T *pzp = plane_ptr(pz.slot);
    const T *ptp = plane_ptr(pt.slot);
#pragma unroll
    for (int r = 0; r < VY; r++) vt[r] = lds16(ptp + rc0 + r * BX);
    const Vec16<T> vn = lds16(pzp + rc0 - BX);
    const Vec16<T> vs = lds16(pzp + rc0 + VY * BX);
    T wl[VY], er[VY];
#pragma unroll
    for (int r = 0; r < VY; r++) {
      wl[r] = pzp[rc0 + r * BX - 1];
      er[r] = pzp[rc0 + r * BX + V];
    }
    release(pz.slot);  // this warp is done with the plane of z
    const bool zedge = !PERIODIC && (z == 0 || z == nz - 1);
    Vec16<T> res[VY];
    if (!(yedge || zedge)) {
#pragma unroll
      for (int r = 0; r < VY; r++)
        res[r] = diff7_row<T, FAST>(kk, vc[r], wl[r], er[r], r == 0 ? vn : vc[r - 1],
                                    r == VY - 1 ? vs : vc[r + 1], vb[r], vt[r], xfix);
    } else {
#pragma unroll
      for (int r = 0; r < VY; r++) {
        const Vec16<T> &nv = r == 0 ? vn : vc[r - 1];
        const Vec16<T> &sv = r == VY - 1 ? vs : vc[r + 1];
        const int y = yg0 + r;
#pragma unroll
        for (int v = 0; v < V; v++) {
          const int x = xg0 + v;
          T c = vc[r].v[v];
          T w = v == 0 ? wl[r] : vc[r].v[v - 1];
          T e = v == V - 1 ? er[r] : vc[r].v[v + 1];
          T n = nv.v[v], s = sv.v[v], bb = vb[r].v[v], t = vt[r].v[v];
          if (x == 0) w = c;
          if (x == nx - 1) e = c;
          if (y == 0) n = c;
          if (y == ny - 1) s = c;
          if (z == 0) bb = c;
          if (z == nz - 1) t = c;
          res[r].v[v] = diff7_point<T, FAST>(k, c, w, e, n, s, bb, t);
        }
      }
    }
    if (ACC) {
#pragma unroll
      for (int r = 0; r < VY; r++) {
        if (!row_in[r]) continue;
#pragma unroll
        for (int v = 0; v < V; v++) {
          if (xg0 + v < d.lo[0] || xg0 + v >= d.hi[0]) continue;
          const double nv = (double)res[r].v[v], dv = nv - (double)vc[r].v[v];
          acc->a += dv * dv;
          acc->b += nv * nv;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < VY; r++) {
      if (!row_in[r]) continue;
      T *dst = dst0 + r * out.sy;
      store_vec(dst, res[r]);
      if (PERIODIC && images) {
        const int y = yg0 + r;
        if (img_x0) dst[nx] = res[r].v[0];
        if (img_x1) {
#pragma unroll
          for (int v = 0; v < V; v++)
            if (v == vlast) dst[v - nx] = res[r].v[v];
        }
        if (y == 0) store_vec(dst + (int64_t)ny * out.sy, res[r]);
        if (y == ny - 1) store_vec(dst - (int64_t)ny * out.sy, res[r]);
        if (z == 0) store_vec(dst + (int64_t)nz * out.sz, res[r]);
        if (z == nz - 1) store_vec(dst - (int64_t)nz * out.sz, res[r]);
      }
    }
    dst0 += out.sz;
    pz = pt;
    z++;
    return true;
  };

  // Prologue: planes 0 (z-1) and 1 (z).
  Vec16<T> A[VY], B[VY], C[VY];
  bool bad = !wait_plane(p);
  bad = bad || !wait_plane(pz);
  if (!bad) {
    const T *p0 = plane_ptr(p.slot), *p1 = plane_ptr(pz.slot);
#pragma unroll
    for (int r = 0; r < VY; r++) {
      A[r] = lds16(p0 + rc0 + r * BX);
      B[r] = lds16(p1 + rc0 + r * BX);
    }
    release(p.slot);
    // Three steps per trip rotate the register roles (b, c, t) without moves.
    int jj = 0;
    for (; jj + 3 <= nzl; jj += 3) {
      if (!step(A, B, C) || !step(B, C, A) || !step(C, A, B)) {
        bad = true;
        break;
      }
    }
    if (!bad && jj < nzl) {
      bad = !step(A, B, C);
      if (!bad && jj + 1 < nzl) bad = !step(B, C, A);
    }
  }
  if (bad) return false;
  // The last plane (z+1 of the last output plane) was never a plane of z.
  release(pt.slot);
  p = pt;
  ring_next(p, S);
  return true;
}

// --------------------------------------------------------------------------
// Temporal blocking, depth 2 (float, clamped faces)
//
// One pass advances two time steps. Per CTA: a producer thread streams input
// planes (box 144 x 20: the 128 x 16 output tile with a 2-cell halo, x
// rounded out to 16 bytes) into ring R1; the "stage-1" warps compute the
// intermediate step over the tile plus a 1-cell halo (130 x 18 points, each
// row as 32 vectors plus two edge scalars) into ring R2, whose stages have
// exactly the layout of a 136 x 18 input box of the output tile (18 / VY1
// stage-1 warps, VY1 rows each); eight
// "stage-2" warps run the ordinary consumer (diff7_consume) on R2. Every
// point of both steps is computed with the single-step arithmetic and face
// rules, so results are bit-identical to two separate steps; intermediate
// values outside the grid are never read (clamped faces select the point
// itself instead).
// --------------------------------------------------------------------------
constexpr int kTbTX = 128, kTbTY = 16;
constexpr int kTbBX1 = kTbTX + 16, kTbBY1 = kTbTY + 4;   // input box
constexpr int kTbBX2 = kTbTX + 8, kTbBY2 = kTbTY + 2;    // intermediate plane
#ifndef PSB_TB_VY1
#define PSB_TB_VY1 2
#endif
constexpr int kTbVY1 = PSB_TB_VY1;                 // intermediate rows per stage-1 thread
constexpr int kTbS1Warps = kTbBY2 / kTbVY1, kTbS2Warps = 8;
constexpr int kTbThreads = 32 + 32 * kTbS1Warps + 32 * kTbS2Warps;

// Stage 1: intermediate planes zb-1 .. zb+nzl of the tile at (x0, y0) from
// input planes zb-2 .. zb+nzl+1 (ring R1, all released), written to ring R2
// (this group fills its stages; the stage-2 warps release them). t1 is the
// thread's index in the stage-1 group.
// FAST: the contracted arithmetic of the FMA mode (diff7_row_fast,
// diff7_point<FAST>), as the single-step FMA kernel computes each point.
template <bool FAST = false>
__device__ __forceinline__ bool diff7_tb_stage1(const Ring &R1, RingPos &p1, const Ring &R2,
                                                RingPos &p2, int t1, int nx, int ny, int nz,
                                                const C7<float> k, int x0, int y0, int zb,
                                                int nzl) {
  constexpr int V = 4, VY = kTbVY1;
  constexpr int BX = kTbBX1;
  const int lane = t1 & 31;
  const int tx = t1 & 31, ty = t1 >> 5;  // 32 vector columns x groups of VY rows
  const int xg0 = x0 + tx * V;
  const int ri0 = ty * VY;                // first intermediate row (y = y0 - 1 + ri)
  const int yg0 = y0 - 1 + ri0;
  const int rc0 = (ri0 + 1) * BX + 8 + tx * V;  // input-box offset of (xg0, row ri0)
  const int wc0 = ri0 * kTbBX2 + 4 + tx * V;     // R2 offset of the same point
  // Edge scalars: columns x0-1 and x0+128 of the 18 intermediate rows, one per
  // fifth thread so that every warp takes a few.
  const bool edge = (t1 % 5) == 0 && t1 / 5 < 2 * kTbBY2;
  const int ecol = edge ? (t1 / 5) / kTbBY2 : 0;   // 0: x0 - 1, 1: x0 + 128
  const int erow = edge ? (t1 / 5) % kTbBY2 : 0;
  const int ex = ecol ? x0 + kTbTX : x0 - 1;
  const int ey = y0 - 1 + erow;
  const int erc = (erow + 1) * BX + (ecol ? 8 + kTbTX : 7);
  const int ewc = erow * kTbBX2 + (ecol ? 4 + kTbTX : 3);

  unsigned xfix = 0;
  if (xg0 == 0) xfix |= 16u;
#pragma unroll
  for (int v = 0; v < V; v++)
    if (xg0 + v == nx - 1) xfix |= 1u << v;
  bool yedge = false;
#pragma unroll
  for (int r = 0; r < VY; r++) yedge = yedge || yg0 + r == 0 || yg0 + r == ny - 1;
  const K7<float> kk = make_k7(k);

  auto wait_full = [&](const Ring &R, const RingPos &q) -> bool {
    bool ok = mbar_wait_bounded(&R.full[q.slot], q.round & 1);
    return __all_sync(0xffffffffu, ok);
  };
  auto release = [&](int slot) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&R1.empty[slot]);
  };
  auto plane = [&](int slot) -> const float * {
    return reinterpret_cast<const float *>(R1.base + slot * R1.stage_bytes);
  };

  RingPos pz = p1;
  ring_next(pz, R1.S);
  RingPos pt = pz;
  int z = zb - 1;  // intermediate plane of the current step
  float eb = 0.f, ec = 0.f;

  auto step = [&](Vec16<float>(&vb)[VY], Vec16<float>(&vc)[VY], Vec16<float>(&vt)[VY]) -> bool {
    ring_next(pt, R1.S);
    if (!wait_full(R1, pt)) return false;
    const float *pzp = plane(pz.slot);
    const float *ptp = plane(pt.slot);
#pragma unroll
    for (int r = 0; r < VY; r++) vt[r] = lds16(ptp + rc0 + r * BX);
    const Vec16<float> vn = lds16(pzp + rc0 - BX);
    const Vec16<float> vs = lds16(pzp + rc0 + VY * BX);
    float wl[VY], er[VY];
#pragma unroll
    for (int r = 0; r < VY; r++) {
      wl[r] = pzp[rc0 + r * BX - 1];
      er[r] = pzp[rc0 + r * BX + V];
    }
    float en = 0.f, es = 0.f, ew = 0.f, ee = 0.f, et = 0.f;
    if (edge) {
      et = ptp[erc];
      en = pzp[erc - BX];
      es = pzp[erc + BX];
      ew = pzp[erc - 1];
      ee = pzp[erc + 1];
    }
    release(pz.slot);
    const bool zedge = z == 0 || z == nz - 1;
    Vec16<float> res[VY];
    if (!(yedge || zedge)) {
#pragma unroll
      for (int r = 0; r < VY; r++) {
        if constexpr (FAST)
          res[r] = diff7_row_fast(kk, vc[r], wl[r], er[r], r == 0 ? vn : vc[r - 1],
                                  r == VY - 1 ? vs : vc[r + 1], vb[r], vt[r], xfix);
        else
          res[r] = diff7_row(kk, vc[r], wl[r], er[r], r == 0 ? vn : vc[r - 1],
                             r == VY - 1 ? vs : vc[r + 1], vb[r], vt[r], xfix);
      }
    } else {
#pragma unroll
      for (int r = 0; r < VY; r++) {
        const Vec16<float> &nv = r == 0 ? vn : vc[r - 1];
        const Vec16<float> &sv = r == VY - 1 ? vs : vc[r + 1];
        const int y = yg0 + r;
#pragma unroll
        for (int v = 0; v < V; v++) {
          const int x = xg0 + v;
          float c = vc[r].v[v];
          float w = v == 0 ? wl[r] : vc[r].v[v - 1];
          float e = v == V - 1 ? er[r] : vc[r].v[v + 1];
          float n = nv.v[v], s = sv.v[v], bb = vb[r].v[v], t = vt[r].v[v];
          if (x == 0) w = c;
          if (x == nx - 1) e = c;
          if (y == 0) n = c;
          if (y == ny - 1) s = c;
          if (z == 0) bb = c;
          if (z == nz - 1) t = c;
          res[r].v[v] = diff7_point<float, FAST>(k, c, w, e, n, s, bb, t);
        }
      }
    }
    float eres = 0.f;
    if (edge) {
      float w = ew, e = ee, n = en, s = es, bb = eb, t = et;
      if (ex == 0) w = ec;
      if (ex == nx - 1) e = ec;
      if (ey == 0) n = ec;
      if (ey == ny - 1) s = ec;
      if (z == 0) bb = ec;
      if (z == nz - 1) t = ec;
      eres = diff7_point<float, FAST>(k, ec, w, e, n, s, bb, t);
      eb = ec;
      ec = et;
    }
    // The intermediate plane into the next stage of R2.
    if (p2.round > 0 && !__all_sync(0xffffffffu, mbar_wait_bounded(&R2.empty[p2.slot],
                                                                   (p2.round - 1) & 1)))
      return false;
    float *dst = reinterpret_cast<float *>(R2.base + p2.slot * R2.stage_bytes);
#pragma unroll
    for (int r = 0; r < VY; r++)
      *reinterpret_cast<float4 *>(dst + wc0 + r * kTbBX2) =
          make_float4(res[r].v[0], res[r].v[1], res[r].v[2], res[r].v[3]);
    if (edge) dst[ewc] = eres;
    __syncwarp();
    if (lane == 0) mbar_arrive(&R2.full[p2.slot]);
    ring_next(p2, R2.S);
    pz = pt;
    z++;
    return true;
  };

  const int nsteps = nzl + 2;
  Vec16<float> A[VY], B[VY], C[VY];
  bool bad = !wait_full(R1, p1);
  bad = bad || !wait_full(R1, pz);
  if (!bad) {
    const float *q0 = plane(p1.slot), *q1 = plane(pz.slot);
#pragma unroll
    for (int r = 0; r < VY; r++) {
      A[r] = lds16(q0 + rc0 + r * BX);
      B[r] = lds16(q1 + rc0 + r * BX);
    }
    if (edge) {
      eb = q0[erc];
      ec = q1[erc];
    }
    release(p1.slot);
    int jj = 0;
    for (; jj + 3 <= nsteps; jj += 3) {
      if (!step(A, B, C) || !step(B, C, A) || !step(C, A, B)) {
        bad = true;
        break;
      }
    }
    if (!bad && jj < nsteps) {
      bad = !step(A, B, C);
      if (!bad && jj + 1 < nsteps) bad = !step(B, C, A);
    }
  }
  if (bad) return false;
  release(pt.slot);
  p1 = pt;
  ring_next(p1, R1.S);
  return true;
}

// One tile as a whole CTA (single-grid kernels): the (TX x TY) column at
// (tile_x, tile_y) of the domain over z chunk zc, read through tensor map
// `tin`, written to `out`. Called by every thread of the CTA; `smem` is the
// CTA's 128-byte aligned dynamic shared memory (barriers + ring).
template <typename T, bool PERIODIC, bool ACC, bool FAST = false>
__device__ __forceinline__ void diff7_tile(const CUtensorMap *tin, const GridView out, int nx,
                                           int ny, int nz, const Dom3 d, const C7<T> k,
                                           const TmaGeom geo, int tile_x, int tile_y, int zc,
                                           int images, int *err, unsigned char *smem,
                                           TileAcc *acc) {
  // The descriptors arrive by value so that they live in registers: callers
  // may pass fields of a table in global memory, and references into it
  // would be reloaded after every store of the hot loop.
  constexpr int V = 16 / sizeof(T);
  const Ring R{reinterpret_cast<uint64_t *>(smem), reinterpret_cast<uint64_t *>(smem) + 32,
               smem + 512, geo.stages, geo.stage_bytes};
  const int nct = geo.tx_threads * geo.ty_threads;  // consumer threads
  const int TX = geo.tx_threads * V, TY = geo.ty_threads * kVY;
  const int x0 = geo.x_base + tile_x * TX;
  const int y0 = d.lo[1] + tile_y * TY;
  const int zb = d.lo[2] + zc * geo.zchunk;
  const int nzl = min(zb + geo.zchunk, d.hi[2]) - zb;  // output planes
  const int tid = threadIdx.x;

  if (tid == 0) ring_init(R, nct >> 5);
  __syncthreads();

  RingPos pos{0, 0};
  if (tid >= nct) {
    if (tid != nct) return;
    tma_prefetch_desc(tin);
    const uint32_t bytes = (uint32_t)(geo.bx * geo.by * sizeof(T));
    if (!ring_produce(R, pos, tin, bytes, x0 - V + geo.ax0, y0 - 1 + geo.ay0, zb - 1 + geo.az0,
                      nzl + 2)) {
      atomicExch(err, 1);
      ring_drain(R, pos);
    }
    return;
  }
  if (!diff7_consume<T, PERIODIC, ACC, FAST>(R, pos, out, nx, ny, nz, d, k, geo, x0, y0, zb, nzl,
                                             images, acc) &&
      (tid & 31) == 0)
    atomicExch(err, 1);
}

}  // namespace psb
