// Device side of the generic stencil on the TMA plane pipeline: the term
// table's device form, the row cache of the packed form, the term programs
// and the kernel body. Included by k_generic_tma.cu (the library's kernel,
// which interprets the table) and by the source of the kernels compiled at
// run time for one table (gt_jit in k_generic_tma.cu), so it includes only
// device.cuh and compiles under the run-time compiler.
#pragma once

#include "device.cuh"

namespace psb {

constexpr int kGtMaxGrids = 4;   // distinct grids read through TMA
constexpr int kGtR = 2;          // largest |offset| per axis (the pitched halo)
#ifndef PSB_GT_VY
#define PSB_GT_VY 4
#endif
// Products of the packed form: 2 all through the f32x2 multiply, 1 only at
// even window offsets (whose pairs of values sit in aligned register pairs),
// 0 scalar. The results are the same; on the 27-point table 1 measured
// fastest (132.0 GLUPS against 130.6 and 128.8).
#ifndef PSB_GT_PACKED_MUL
#define PSB_GT_PACKED_MUL 1
#endif
constexpr int kGtVY = PSB_GT_VY;  // rows per consumer thread
constexpr int kGtConsumers = 128;
constexpr int kGtThreads = kGtConsumers + 32;

// One factor of the device table. kind 0: the constant c; 1: the constant 1
// (no multiply); 2: a staged read at element `off` of the stage of window
// plane k (off = grid index * plane elements + dy * box width + dx).
struct GtFactor {
  int kind;
  int k;
  int off;
  int pad;
  double c;
};

struct GtTable {
  int nterms;
  int has_post;
  GtFactor post;
  GtFactor a[PSB_MAX_TERMS];
  GtFactor b[PSB_MAX_TERMS];
  // Every term one staged read times a constant (the common user stencil),
  // no post factor: a packed form. word = (row offset << 10) | (the run of
  // terms on this row needs the previous lane's values) << 9 | (... the next
  // lane's) << 8 | (coefficient is 1) << 7 | (first term of a run on a new
  // row) << 6 | (dx + 2) << 3 | window plane. The row offset is the read's
  // offset without its x part (a multiple of V): consecutive terms on the
  // same row (same plane, grid and dy) reuse the row's values in registers,
  // and x offsets shift them between lanes with warp shuffles.
  int simple;
  int word[PSB_MAX_TERMS];
  double coef[PSB_MAX_TERMS];    // the constant factor in double grids' arithmetic
  float coef32[PSB_MAX_TERMS];   // ... converted to float once, for float grids
  // Point-wise programs (stencil functions compiled by the DSL front end):
  // the staged grid of each of the function's grid parameters (-1: not
  // read) and the parameters' extents; `coef` holds the scalar arguments.
  int slot_grid[PSB_MAX_GRIDS];
  int slot_dims[PSB_MAX_GRIDS][3];
  // The word a checked read outside its grid sets to PSB_ERR_BOUNDS.
  int *read_err;
};

struct GtMaps {
  CUtensorMap m[kGtMaxGrids];
};

struct GtGeom {
  int ax0[kGtMaxGrids], ay0[kGtMaxGrids], az0[kGtMaxGrids];  // tensor coords of logical 0
  int ngrids;        // box planes per stage
  int bx, by;        // box (elements)
  int plane_elems;   // elements between the grids' planes in a stage
  int stage_bytes;
  int stages;
  int zmin, window;  // first z offset, planes live per output plane
  int x_base, tiles_x, tiles_y, zchunk;
  int tx_threads;    // consumer threads along x (32)
  int vec_store;     // 16-byte stores allowed (aligned output rows)
};

// The VY x V values of one factor for a thread's points, in registers.
template <typename T>
struct GtBlk {
  T v[kGtVY][16 / sizeof(T)];
};

template <typename T>
__device__ __forceinline__ GtBlk<T> gt_load(int kind, int k, int off, double c,
                                            const unsigned char *ring, int sbytes, int S,
                                            int slot0, int thr_off, int bx) {
  constexpr int V = 16 / sizeof(T);
  GtBlk<T> out;
  if (kind != 2) {
    const T cv = kind == 1 ? (T)1 : (T)c;
#pragma unroll
    for (int r = 0; r < kGtVY; r++)
#pragma unroll
      for (int v = 0; v < V; v++) out.v[r][v] = cv;
    return out;
  }
  int s = slot0 + k;
  if (s >= S) s -= S;
  const T *p = reinterpret_cast<const T *>(ring + (size_t)s * sbytes) + off + thr_off;
#pragma unroll
  for (int r = 0; r < kGtVY; r++)
#pragma unroll
    for (int v = 0; v < V; v++) out.v[r][v] = p[r * bx + v];
  return out;
}

// The values of one staged row around a thread's V points: its own aligned
// vector a (x .. x+V-1), the first two values after it (the next lane's, or
// loaded by the last lane) and the two before it (the previous lane's, or
// loaded by lane 0): ext = [p0 p1 a0 .. aV-1 n0 n1], so the term at x offset
// dx takes ext[2 + dx + j] for its point j.
template <typename T>
struct GtRow {
  T e[16 / sizeof(T) + 4];
};

template <typename T>
__device__ __forceinline__ void gt_row_load(const T *p, int lane, bool need_n, bool need_p,
                                            GtRow<T> &r) {
  constexpr int V = 16 / sizeof(T);
  const Vec16<T> a = lds16(p);
#pragma unroll
  for (int j = 0; j < V; j++) r.e[2 + j] = a.v[j];
  if (need_n) {
    r.e[V + 2] = __shfl_down_sync(0xffffffffu, a.v[0], 1);
    r.e[V + 3] = __shfl_down_sync(0xffffffffu, a.v[1], 1);
    if (lane == 31) {
      r.e[V + 2] = p[V];
      r.e[V + 3] = p[V + 1];
    }
  }
  if (need_p) {
    r.e[0] = __shfl_up_sync(0xffffffffu, a.v[V - 2], 1);
    r.e[1] = __shfl_up_sync(0xffffffffu, a.v[V - 1], 1);
    if (lane == 0) {
      r.e[0] = p[-2];
      r.e[1] = p[-1];
    }
  }
}

// One packed-form term on the cached rows: the window ext[DXP2 + j] (x
// offset DXP2 - 2), times c unless ONE, added to the running sum (FIRST:
// starts it, as the reference's sum starts from its first term). Float
// products go in pairs through the sm_100 f32x2 multiply (each lane rounded
// like the scalar one); the sums stay scalar. FMA (the contracted arithmetic
// mode, compiled kernels only): a term after the first is added with one
// rounding, c * x + sum fused (paired for float); the first product and
// unmultiplied terms round as in the exact form.
template <int DXP2, bool ONE, bool FIRST, bool FMA = false>
__device__ __forceinline__ void gt_term(const GtRow<float> (&row)[kGtVY], float c,
                                        GtBlk<float> &acc) {
  const float2 cc = make_float2(c, c);
#pragma unroll
  for (int r = 0; r < kGtVY; r++) {
    float2 lo = make_float2(row[r].e[DXP2], row[r].e[DXP2 + 1]);
    float2 hi = make_float2(row[r].e[DXP2 + 2], row[r].e[DXP2 + 3]);
    if (FMA && !FIRST && !ONE) {
      // The contracted form: acc + c * x with one rounding (paired).
      const float2 a = __ffma2_rn(cc, lo, make_float2(acc.v[r][0], acc.v[r][1]));
      const float2 b = __ffma2_rn(cc, hi, make_float2(acc.v[r][2], acc.v[r][3]));
      acc.v[r][0] = a.x;
      acc.v[r][1] = a.y;
      acc.v[r][2] = b.x;
      acc.v[r][3] = b.y;
      continue;
    }
    if (!ONE) {
      if (PSB_GT_PACKED_MUL == 2 || (PSB_GT_PACKED_MUL == 1 && DXP2 % 2 == 0)) {
        lo = __fmul2_rn(cc, lo);
        hi = __fmul2_rn(cc, hi);
      } else {
        lo = make_float2(xmul(c, lo.x), xmul(c, lo.y));
        hi = make_float2(xmul(c, hi.x), xmul(c, hi.y));
      }
    }
    if (FIRST) {
      acc.v[r][0] = lo.x;
      acc.v[r][1] = lo.y;
      acc.v[r][2] = hi.x;
      acc.v[r][3] = hi.y;
    } else {  // scalar adds: paired f32x2 adds gave results 1 ulp off the scalar sums
      acc.v[r][0] = xadd(acc.v[r][0], lo.x);
      acc.v[r][1] = xadd(acc.v[r][1], lo.y);
      acc.v[r][2] = xadd(acc.v[r][2], hi.x);
      acc.v[r][3] = xadd(acc.v[r][3], hi.y);
    }
  }
}

template <int DXP2, bool ONE, bool FIRST, bool FMA = false>
__device__ __forceinline__ void gt_term(const GtRow<double> (&row)[kGtVY], double c,
                                        GtBlk<double> &acc) {
#pragma unroll
  for (int r = 0; r < kGtVY; r++)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      double v = row[r].e[DXP2 + j];
      if (FMA && !FIRST && !ONE) {
        acc.v[r][j] = __fma_rn(c, v, acc.v[r][j]);
        continue;
      }
      if (!ONE) v = xmul(c, v);
      acc.v[r][j] = FIRST ? v : xadd(acc.v[r][j], v);
    }
}

// key = (dx + 2) | (coefficient is 1) << 3, uniform across the warp.
template <bool FIRST, typename T>
__device__ __forceinline__ void gt_term_key(int key, const GtRow<T> (&row)[kGtVY], T c,
                                            GtBlk<T> &acc) {
  switch (key) {
    case 0: gt_term<0, false, FIRST>(row, c, acc); break;
    case 1: gt_term<1, false, FIRST>(row, c, acc); break;
    case 2: gt_term<2, false, FIRST>(row, c, acc); break;
    case 3: gt_term<3, false, FIRST>(row, c, acc); break;
    case 4: gt_term<4, false, FIRST>(row, c, acc); break;
    case 8: gt_term<0, true, FIRST>(row, c, acc); break;
    case 9: gt_term<1, true, FIRST>(row, c, acc); break;
    case 10: gt_term<2, true, FIRST>(row, c, acc); break;
    case 11: gt_term<3, true, FIRST>(row, c, acc); break;
    default: gt_term<4, true, FIRST>(row, c, acc); break;
  }
}

__device__ __forceinline__ float gt_coef(const GtTable &tab, int t, float) {
  return tab.coef32[t];
}
__device__ __forceinline__ double gt_coef(const GtTable &tab, int t, double) {
  return tab.coef[t];
}

// One term of the general form, a_t * b_t (b_t = 1: a_t alone), added to
// the running sum (first: starts it). The interpreting kernel passes the
// table's factors; a compiled kernel passes factors whose kind, plane and
// offset are constants, so the loads fold to fixed shared-memory offsets.
template <typename T>
__device__ __forceinline__ void gt_general_term(const GtFactor &fa, const GtFactor &fb,
                                                bool first, const unsigned char *ring,
                                                int sbytes, int S, int slot0, int thr_off,
                                                int bx, GtBlk<T> &acc) {
  constexpr int V = 16 / sizeof(T);
  const GtBlk<T> va = gt_load<T>(fa.kind, fa.k, fa.off, fa.c, ring, sbytes, S, slot0, thr_off, bx);
  GtBlk<T> p = va;
  if (fb.kind != 1) {
    const GtBlk<T> vb =
        gt_load<T>(fb.kind, fb.k, fb.off, fb.c, ring, sbytes, S, slot0, thr_off, bx);
#pragma unroll
    for (int r = 0; r < kGtVY; r++)
#pragma unroll
      for (int v = 0; v < V; v++) p.v[r][v] = xmul(va.v[r][v], vb.v[r][v]);
  }
  if (first) {
    acc = p;
  } else {
#pragma unroll
    for (int r = 0; r < kGtVY; r++)
#pragma unroll
      for (int v = 0; v < V; v++) acc.v[r][v] = xadd(acc.v[r][v], p.v[r][v]);
  }
}

__device__ __forceinline__ int gt_key(int w) { return ((w >> 3) & 7) | ((w >> 4) & 8); }

// The VY rows of the run that starts with a term word's fields (window
// plane k, row offset), with the neighbouring lanes' values it needs.
template <typename T>
__device__ __forceinline__ void gt_rows(const unsigned char *ring, int sbytes, int S, int slot0,
                                        int thr_off, int bx, int lane, int k, int rowoff,
                                        bool need_n, bool need_p, GtRow<T> (&row)[kGtVY]) {
  int sl = slot0 + k;
  if (sl >= S) sl -= S;
  const T *p = reinterpret_cast<const T *>(ring + (size_t)sl * sbytes) + rowoff + thr_off;
#pragma unroll
  for (int r = 0; r < kGtVY; r++) gt_row_load(p + r * bx, lane, need_n, need_p, row[r]);
}

// Where a consumer thread's block of points sits in the window of staged
// planes, for point-wise programs: the thread's first point (x, y, z), its
// offset in a stage (thr_off) and the ring's geometry.
struct GtAt {
  const unsigned char *ring;
  int sbytes, S, slot0, thr_off, bx, plane_elems, zmin;
  int x, y, z;
  int lo0, hi0, lo1, hi1;  // the domain in x and y (z is always inside)
};

// The staged value of grid slot `slot` at (x + dx, y + dy, z + dz) from the
// point in row r, column v of the thread's block (offsets within the halo
// the window holds).
template <typename T>
__device__ __forceinline__ T gt_staged(const GtTable &tab, const GtAt &at, int slot, int r, int v,
                                       int dx, int dy, int dz) {
  int sl = at.slot0 + dz - at.zmin;
  if (sl >= at.S) sl -= at.S;
  const T *p = reinterpret_cast<const T *>(at.ring + (size_t)sl * at.sbytes);
  return p[tab.slot_grid[slot] * at.plane_elems + at.thr_off + (r + dy) * at.bx + v + dx];
}

// The library's term program: reads the packed table word by word.
struct GtTableProg {
  static constexpr bool kCompiled = false;
  static constexpr bool kPoints = false;
  template <typename T>
  static __device__ __forceinline__ void eval(const GtTable &tab, const unsigned char *ring,
                                              int sbytes, int S, int slot0, int thr_off, int bx,
                                              int lane, GtBlk<T> &acc) {
    GtRow<T> row[kGtVY];
    const int w0 = tab.word[0];
    gt_rows<T>(ring, sbytes, S, slot0, thr_off, bx, lane, w0 & 7, w0 >> 10, (w0 >> 8) & 1,
               (w0 >> 9) & 1, row);
    gt_term_key<true>(gt_key(w0), row, gt_coef(tab, 0, T()), acc);
    for (int t = 1; t < tab.nterms; t++) {
      const int w = tab.word[t];
      if (w & 64)  // a new row: its values into registers
        gt_rows<T>(ring, sbytes, S, slot0, thr_off, bx, lane, w & 7, w >> 10, (w >> 8) & 1,
                   (w >> 9) & 1, row);
      gt_term_key<false>(gt_key(w), row, gt_coef(tab, t, T()), acc);
    }
  }
};

// The kernel body, shared by the library's own kernel (which interprets the
// term table) and kernels compiled at run time for one table (whose term
// program is fixed at compile time). Prog::eval evaluates the sum of the
// terms; the library's program handles packed tables only (general ones take
// the loop below), a compiled program (Prog::kCompiled) is the whole table,
// packed or general. The post factor is applied here in both cases. A
// point-wise program (Prog::kPoints: a compiled stencil function) computes
// each point of the thread's block itself from the staged window
// (gt_staged) and emits into acc.
template <typename T, class Prog>
__device__ __forceinline__ void gt_body(const GtMaps &maps, const GtTable &tab,
                                        const GridView &out, const Dom3 &d, const GtGeom &geo,
                                        int *err) {
  constexpr int V = 16 / sizeof(T);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *empty = full + 32;
  unsigned char *ring = smem + 512;
  const int S = geo.stages, W = geo.window;
  const int TX = geo.tx_threads * V, TY = (kGtConsumers / geo.tx_threads) * kGtVY;
  int b = blockIdx.x;
  const int tile_x = b % geo.tiles_x;
  b /= geo.tiles_x;
  const int tile_y = b % geo.tiles_y;
  const int zc = b / geo.tiles_y;
  const int x0 = geo.x_base + tile_x * TX;
  const int y0 = d.lo[1] + tile_y * TY;
  const int zb = d.lo[2] + zc * geo.zchunk;
  const int nzl = min(zb + geo.zchunk, d.hi[2]) - zb;
  const int nplanes = nzl + W - 1;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int i = 0; i < S; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], kGtConsumers / 32);
    }
    mbar_fence_init();
  }
  __syncthreads();

  if (tid >= kGtConsumers) {
    // Producer: input plane j (z = zb + zmin + j) of every grid into stage j % S.
    if (tid != kGtConsumers) return;
    for (int g = 0; g < geo.ngrids; g++) tma_prefetch_desc(&maps.m[g]);
    const uint32_t bytes = (uint32_t)(geo.ngrids * geo.bx * geo.by * sizeof(T));
    for (int j = 0; j < nplanes; j++) {
      const int slot = j % S;
      if (j >= S && !mbar_wait_bounded(&empty[slot], ((j / S) - 1) & 1)) {
        atomicExch(err, 1);
        ring_drain(Ring{full, empty, ring, S, geo.stage_bytes}, RingPos{slot, (uint32_t)(j / S)});
        return;
      }
      mbar_arrive_expect_tx(&full[slot], bytes);
      const int z = zb + geo.zmin + j;
      unsigned char *dst = ring + (size_t)slot * geo.stage_bytes;
      for (int g = 0; g < geo.ngrids; g++)
        tma_load_3d(dst + (size_t)g * geo.plane_elems * sizeof(T), &maps.m[g], &full[slot],
                    x0 - V + geo.ax0[g], y0 - kGtR + geo.ay0[g], z + geo.az0[g]);
    }
    return;
  }

  // Consumers.
  const int lane = tid & 31;
  const int tx = tid % geo.tx_threads, ty = tid / geo.tx_threads;
  const int xg0 = x0 + tx * V, yg0 = y0 + ty * kGtVY;
  const int thr_off = (ty * kGtVY + kGtR) * geo.bx + V + tx * V;
  const bool xvec = geo.vec_store && xg0 >= d.lo[0] && xg0 + V <= d.hi[0];
  bool row_in[kGtVY];
#pragma unroll
  for (int r = 0; r < kGtVY; r++) row_in[r] = yg0 + r >= d.lo[1] && yg0 + r < d.hi[1];
  T *o = (T *)out.origin;

  auto wait_full = [&](int j) -> bool {
    const bool ok = mbar_wait_bounded(&full[j % S], (j / S) & 1);
    return __all_sync(0xffffffffu, ok);
  };
  auto release = [&](int j) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[j % S]);
  };

  bool bad = false;
  for (int j = 0; j < W - 1 && !bad; j++) bad = !wait_full(j);
  for (int i = 0; i < nzl && !bad; i++) {
    if (!wait_full(i + W - 1)) {
      bad = true;
      break;
    }
    const int slot0 = i % S;
    GtBlk<T> acc;
    if constexpr (Prog::kPoints) {
      const GtAt at{ring, geo.stage_bytes, S, slot0, thr_off, geo.bx, geo.plane_elems, geo.zmin,
                    xg0, yg0, zb + i, d.lo[0], d.hi[0], d.lo[1], d.hi[1]};
      Prog::template eval_points<T>(tab, at, acc);
    } else if (Prog::kCompiled || tab.simple) {
      Prog::template eval<T>(tab, ring, geo.stage_bytes, S, slot0, thr_off, geo.bx, lane, acc);
    } else {
      for (int t = 0; t < tab.nterms; t++)
        gt_general_term<T>(tab.a[t], tab.b[t], t == 0, ring, geo.stage_bytes, S, slot0, thr_off,
                           geo.bx, acc);
    }
    if (tab.has_post) {
      const GtFactor fp = tab.post;
      const GtBlk<T> vp = gt_load<T>(fp.kind, fp.k, fp.off, fp.c, ring, geo.stage_bytes, S,
                                     slot0, thr_off, geo.bx);
#pragma unroll
      for (int r = 0; r < kGtVY; r++)
#pragma unroll
        for (int v = 0; v < V; v++) acc.v[r][v] = xmul(acc.v[r][v], vp.v[r][v]);
    }
    release(i);  // input plane zb + zmin + i is not read by later output planes
    const int z = zb + i;
#pragma unroll
    for (int r = 0; r < kGtVY; r++) {
      if (!row_in[r]) continue;
      T *dst = o + (int64_t)xg0 + (int64_t)(yg0 + r) * out.sy + (int64_t)z * out.sz;
      if (xvec) {
        Vec16<T> w;
#pragma unroll
        for (int v = 0; v < V; v++) w.v[v] = acc.v[r][v];
        stg16(dst, w);
      } else {
#pragma unroll
        for (int v = 0; v < V; v++)
          if (xg0 + v >= d.lo[0] && xg0 + v < d.hi[0]) dst[v] = acc.v[r][v];
      }
    }
  }
  if (bad) {
    if (lane == 0) atomicExch(err, 1);
    return;
  }
  for (int j = nzl; j < nplanes; j++) release(j);
}

}  // namespace psb
