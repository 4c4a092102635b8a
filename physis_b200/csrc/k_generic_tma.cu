// Generic flat linear stencil on the TMA plane pipeline (2.5-D z-streaming).
//
// The B200 path for user stencils registered as psb_generic_stencil (the
// executable form of the reference's flat-sum stencil functions,
// tests/system_tests/test_cases/test_*.c, which its CUDA target turns into
// one-thread-per-(x,y) kernels with a z loop and global loads,
// translator/cuda_translator.cc:615-869). Here each CTA owns a TX x TY
// column of the domain and a chunk of z. A producer thread streams, for
// every input plane, one TMA box of each grid the stencil reads -- the tile
// plus the halo the term table's offsets need (|offset| <= 2 per axis) --
// into a ring of shared-memory stages; the z offsets of the table set how
// many planes are live at once (a window of zmax - zmin + 1 stages), so
// every input plane is read from HBM once per tile. Consumer warps evaluate
// the term table on the staged planes: each thread owns V consecutive x
// points (16 bytes) of VY rows, reads every factor from shared memory and
// stores 16 bytes at a time.
//
// Arithmetic and order are those of k_generic (and of the reference's CPU
// target): each term a_i * b_i rounded in the accumulation type, summed left
// to right, times the optional post factor; a factor that is the constant 1
// is not multiplied (x * 1 == x exactly). Results are bit-identical to the
// thread-per-point kernel.
//
// Boundary forms: plain reads take the grid's own cells (the map was checked
// to stay inside the grid); periodic and clamped reads take the resident
// halo of a pitched grid, which the launcher refreshes with the periodic or
// clamped image of the interior (k_halo_fill) whenever the grid changed
// since. A grid read both ways, an in-place map, red-black order, lower-
// dimensional or mixed-type grids, and offsets beyond the halo use k_generic.
#include <algorithm>
#include <cstring>

#include "k_generic.cuh"

namespace psb {

constexpr int kGtMaxGrids = 4;   // distinct grids read through TMA
constexpr int kGtR = 2;          // largest |offset| per axis (the pitched halo)
#ifndef PSB_GT_VY
#define PSB_GT_VY 4
#endif
// Products of the packed form: 2 all through the f32x2 multiply, 1 only at
// even window offsets, 0 scalar (the results are the same; the instruction
// counts differ).
#ifndef PSB_GT_PACKED_MUL
#define PSB_GT_PACKED_MUL 2
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
// like the scalar one); the sums stay scalar.
template <int DXP2, bool ONE, bool FIRST>
__device__ __forceinline__ void gt_term(const GtRow<float> (&row)[kGtVY], float c,
                                        GtBlk<float> &acc) {
  const float2 cc = make_float2(c, c);
#pragma unroll
  for (int r = 0; r < kGtVY; r++) {
    float2 lo = make_float2(row[r].e[DXP2], row[r].e[DXP2 + 1]);
    float2 hi = make_float2(row[r].e[DXP2 + 2], row[r].e[DXP2 + 3]);
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
    } else {  // scalar adds: a packed add may be fused with the packed multiply
      acc.v[r][0] = xadd(acc.v[r][0], lo.x);
      acc.v[r][1] = xadd(acc.v[r][1], lo.y);
      acc.v[r][2] = xadd(acc.v[r][2], hi.x);
      acc.v[r][3] = xadd(acc.v[r][3], hi.y);
    }
  }
}

template <int DXP2, bool ONE, bool FIRST>
__device__ __forceinline__ void gt_term(const GtRow<double> (&row)[kGtVY], double c,
                                        GtBlk<double> &acc) {
#pragma unroll
  for (int r = 0; r < kGtVY; r++)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      double v = row[r].e[DXP2 + j];
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

// c times the V values of a row, each product rounded (packed for float).
__device__ __forceinline__ void gt_scale(float c, float (&o)[4]) {
  const float2 cc = make_float2(c, c);
  const float2 lo = __fmul2_rn(cc, make_float2(o[0], o[1]));
  const float2 hi = __fmul2_rn(cc, make_float2(o[2], o[3]));
  o[0] = lo.x; o[1] = lo.y; o[2] = hi.x; o[3] = hi.y;
}

__device__ __forceinline__ void gt_scale(double c, double (&o)[2]) {
  o[0] = xmul(c, o[0]);
  o[1] = xmul(c, o[1]);
}

template <typename T>
__global__ void __launch_bounds__(kGtThreads, sizeof(T) == 4 ? 4 : 3) k_generic_tma(const __grid_constant__ GtMaps maps,
                                                            const __grid_constant__ GtTable tab,
                                                            GridView out, Dom3 d,
                                                            const __grid_constant__ GtGeom geo,
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
    if (tab.simple) {
      GtRow<T> row[kGtVY];
      auto load_rows = [&](int w) {
        int sl = slot0 + (w & 7);
        if (sl >= S) sl -= S;
        const T *p = reinterpret_cast<const T *>(ring + (size_t)sl * geo.stage_bytes) +
                     (w >> 10) + thr_off;
#pragma unroll
        for (int r = 0; r < kGtVY; r++)
          gt_row_load(p + r * geo.bx, lane, (w >> 8) & 1, (w >> 9) & 1, row[r]);
      };
      const int w0 = tab.word[0];
      load_rows(w0);
      gt_term_key<true>(((w0 >> 3) & 7) | ((w0 >> 4) & 8), row, gt_coef(tab, 0, T()), acc);
      for (int t = 1; t < tab.nterms; t++) {
        const int w = tab.word[t];
        if (w & 64) load_rows(w);  // a new row: its values into registers
        gt_term_key<false>(((w >> 3) & 7) | ((w >> 4) & 8), row, gt_coef(tab, t, T()), acc);
      }
    } else {
    for (int t = 0; t < tab.nterms; t++) {
      const GtFactor fa = tab.a[t], fb = tab.b[t];
      const GtBlk<T> va = gt_load<T>(fa.kind, fa.k, fa.off, fa.c, ring, geo.stage_bytes, S,
                                     slot0, thr_off, geo.bx);
      GtBlk<T> p = va;
      if (fb.kind != 1) {
        const GtBlk<T> vb = gt_load<T>(fb.kind, fb.k, fb.off, fb.c, ring, geo.stage_bytes, S,
                                       slot0, thr_off, geo.bx);
#pragma unroll
        for (int r = 0; r < kGtVY; r++)
#pragma unroll
          for (int v = 0; v < V; v++) p.v[r][v] = xmul(va.v[r][v], vb.v[r][v]);
      }
      if (t == 0) {
        acc = p;
      } else {
#pragma unroll
        for (int r = 0; r < kGtVY; r++)
#pragma unroll
          for (int v = 0; v < V; v++) acc.v[r][v] = xadd(acc.v[r][v], p.v[r][v]);
      }
    }
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

// Host: decide whether the map runs on the TMA path and build its table.
struct GtPlan {
  int ngrids = 0;
  int slots[kGtMaxGrids];     // stencil grid slot of each staged grid
  int mode[kGtMaxGrids];      // halo form each staged grid needs (NONE: none)
  int zmin = 0, zmax = 0;
};

static bool gt_factor_ok(const psb_generic_stencil &d, const MapImpl &m, const psb_factor &f,
                         GtPlan &p) {
  if (f.grid < 0) return true;
  if (f.grid >= d.ngrids || f.grid == d.out_grid) return false;
  if (d.grid_type[f.grid] != d.accum_type) return false;
  for (int k = 0; k < 3; k++)
    if (d.grid_axes[f.grid][k] != k || f.offset[k] < -kGtR || f.offset[k] > kGtR) return false;
  if (m.grids[f.grid] == m.grids[d.out_grid]) return false;  // in place
  int gi = -1;
  for (int i = 0; i < p.ngrids; i++)
    if (p.slots[i] == f.grid) gi = i;
  if (gi < 0) {
    if (p.ngrids == kGtMaxGrids) return false;
    gi = p.ngrids++;
    p.slots[gi] = f.grid;
    p.mode[gi] = PSB_BOUNDARY_NONE;
  }
  if (f.boundary != PSB_BOUNDARY_NONE) {
    if (p.mode[gi] != PSB_BOUNDARY_NONE && p.mode[gi] != f.boundary) return false;
    if (m.grids[f.grid]->layout != PSB_LAYOUT_PITCHED) return false;
    p.mode[gi] = f.boundary;
  }
  p.zmin = std::min(p.zmin, f.offset[2]);
  p.zmax = std::max(p.zmax, f.offset[2]);
  return true;
}

static GtFactor gt_compact(const psb_factor &f, const GtPlan &p, int plane_elems, int bx) {
  GtFactor g;
  memset(&g, 0, sizeof(g));
  if (f.grid < 0) {
    g.kind = f.constant == 1.0 ? 1 : 0;
    g.c = f.constant;
    return g;
  }
  int gi = 0;
  for (int i = 0; i < p.ngrids; i++)
    if (p.slots[i] == f.grid) gi = i;
  g.kind = 2;
  g.k = f.offset[2] - p.zmin;
  g.off = gi * plane_elems + f.offset[1] * bx + f.offset[0];
  return g;
}

static int g_last_generic_impl = PSB_IMPL_GENERIC;

template <typename T>
static psb_status gt_launch(MapImpl &m, const psb_generic_stencil &desc, const GtPlan &p,
                            cudaStream_t s, int64_t *launches) {
  constexpr int V = 16 / sizeof(T);
  Runtime &r = rt();
  GridImpl *og = m.grids[desc.out_grid];
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    d.lo[i] = m.dom.local_min[i];
    d.hi[i] = m.dom.local_max[i];
  }
  GtGeom geo;
  memset(&geo, 0, sizeof(geo));
  geo.tx_threads = 32;
  const int TX = geo.tx_threads * V, TY = (kGtConsumers / geo.tx_threads) * kGtVY;
  geo.bx = TX + 2 * V;
  geo.by = TY + 2 * kGtR;
  geo.ngrids = p.ngrids;
  geo.plane_elems = (geo.bx * geo.by * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
  geo.stage_bytes = geo.ngrids * geo.plane_elems * (int)sizeof(T);
  geo.zmin = p.zmin;
  geo.window = p.zmax - p.zmin + 1;
  geo.stages = geo.window + 2;
  geo.x_base = d.lo[0] / V * V;
  geo.tiles_x = (d.hi[0] - geo.x_base + TX - 1) / TX;
  geo.tiles_y = (d.hi[1] - d.lo[1] + TY - 1) / TY;
  geo.vec_store = tma_eligible(og) ? 1 : 0;
  // z chunks: long enough to amortise the window's extra planes, short
  // enough for a few CTAs per SM.
  const int64_t tiles = (int64_t)geo.tiles_x * geo.tiles_y;
  geo.zchunk = 32;
  while (geo.zchunk > 4 && tiles * ((d.hi[2] - d.lo[2] + geo.zchunk - 1) / geo.zchunk) <
                               (int64_t)r.sm_count * 4)
    geo.zchunk /= 2;
  const int nzc = (d.hi[2] - d.lo[2] + geo.zchunk - 1) / geo.zchunk;
  const int64_t nblocks = tiles * nzc;
  if (nblocks > 0x7fffffff) return set_status(PSB_ERR_UNSUPPORTED);
  GtMaps maps;
  memset(&maps, 0, sizeof(maps));
  for (int i = 0; i < p.ngrids; i++) {
    GridImpl *g = m.grids[p.slots[i]];
    const CUtensorMap *tm = nullptr;
    if (get_tmap(g, geo.bx, geo.by, &tm) != PSB_OK) return PSB_ERR_UNSUPPORTED;
    maps.m[i] = *tm;
    const bool pitched = g->layout == PSB_LAYOUT_PITCHED;
    geo.ax0[i] = pitched ? g->pad_left : 0;
    geo.ay0[i] = pitched ? g->halo : 0;
    geo.az0[i] = pitched ? g->halo : 0;
  }
  GtTable tab;
  memset(&tab, 0, sizeof(tab));
  tab.nterms = desc.nterms;
  tab.has_post = desc.has_post;
  for (int t = 0; t < desc.nterms; t++) {
    tab.a[t] = gt_compact(desc.terms[t].a, p, geo.plane_elems, geo.bx);
    tab.b[t] = gt_compact(desc.terms[t].b, p, geo.plane_elems, geo.bx);
  }
  if (desc.has_post) tab.post = gt_compact(desc.post, p, geo.plane_elems, geo.bx);
  // The packed form when every term is one read times a constant.
  tab.simple = !desc.has_post;
  for (int t = 0; t < desc.nterms && tab.simple; t++)
    if ((tab.a[t].kind == 2) == (tab.b[t].kind == 2)) tab.simple = 0;
  if (tab.simple) {
    // Runs of consecutive terms on the same row (plane, grid, dy) share one
    // load; each run records whether it needs the neighbouring lanes.
    int run_start = 0;
    for (int t = 0; t < desc.nterms; t++) {
      const GtFactor &rd = tab.a[t].kind == 2 ? tab.a[t] : tab.b[t];
      const GtFactor &cf = tab.a[t].kind == 2 ? tab.b[t] : tab.a[t];
      const int dx = desc.terms[t].a.grid >= 0 ? desc.terms[t].a.offset[0]
                                               : desc.terms[t].b.offset[0];
      const int rowoff = rd.off - dx;
      const bool fresh = t == 0 || rowoff != (tab.word[t - 1] >> 10) || rd.k != (tab.word[t - 1] & 7);
      if (fresh) run_start = t;
      tab.word[t] = (rowoff << 10) | ((cf.kind == 1) << 7) | (fresh << 6) | ((dx + 2) << 3) | rd.k;
      tab.coef[t] = cf.kind == 1 ? 1.0 : cf.c;
      tab.coef32[t] = (float)tab.coef[t];
      if (dx > 0) tab.word[run_start] |= 1 << 8;
      if (dx < 0) tab.word[run_start] |= 1 << 9;
    }
  }
  const size_t smem = 128 + 512 + (size_t)geo.stages * geo.stage_bytes;
  if (smem > r.smem_optin) return PSB_ERR_UNSUPPORTED;
  static size_t configured[2] = {0, 0};
  size_t &conf = configured[sizeof(T) == 8];
  if (smem > conf) {
    PSB_TRY(cudaFuncSetAttribute(k_generic_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)r.smem_optin));
    PSB_TRY(cudaFuncSetAttribute(k_generic_tma<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    conf = r.smem_optin;
  }
  // Periodic and clamped reads take the halo: refresh it where it is stale.
  for (int i = 0; i < p.ngrids; i++) {
    GridImpl *g = m.grids[p.slots[i]];
    if (p.mode[i] != PSB_BOUNDARY_NONE && g->ghost_valid != p.mode[i])
      PSB_CHECK(launch_halo_fill(g, p.mode[i], s));
  }
  k_generic_tma<T><<<(unsigned)nblocks, kGtThreads, smem, s>>>(maps, tab, og->view(), d, geo,
                                                              r.d_error);
  (*launches)++;
  g_last_generic_impl = PSB_IMPL_TMA;
  return PSB_OK;
}

// PSB_ERR_UNSUPPORTED when the map does not fit the TMA path (the caller
// then runs k_generic).
psb_status generic_tma_launch(MapImpl &m, const GenericDesc &gd, int color, cudaStream_t s,
                              int64_t *launches) {
  const psb_generic_stencil &desc = gd.host;
  g_last_generic_impl = PSB_IMPL_GENERIC;
  if (desc.ndims != 3 || color >= 0 || desc.nterms < 1) return PSB_ERR_UNSUPPORTED;
  if (desc.accum_type != PS_FLOAT && desc.accum_type != PS_DOUBLE) return PSB_ERR_UNSUPPORTED;
  if (desc.grid_type[desc.out_grid] != desc.accum_type) return PSB_ERR_UNSUPPORTED;
  for (int k = 0; k < 3; k++)
    if (desc.grid_axes[desc.out_grid][k] != k) return PSB_ERR_UNSUPPORTED;
  for (int i = 0; i < 3; i++)
    if (m.dom.local_max[i] <= m.dom.local_min[i]) return PSB_ERR_UNSUPPORTED;
  GtPlan p;
  for (int t = 0; t < desc.nterms; t++)
    if (!gt_factor_ok(desc, m, desc.terms[t].a, p) || !gt_factor_ok(desc, m, desc.terms[t].b, p))
      return PSB_ERR_UNSUPPORTED;
  if (desc.has_post && !gt_factor_ok(desc, m, desc.post, p)) return PSB_ERR_UNSUPPORTED;
  if (p.ngrids == 0) return PSB_ERR_UNSUPPORTED;
  for (int i = 0; i < p.ngrids; i++)
    if (!tma_eligible(m.grids[p.slots[i]])) return PSB_ERR_UNSUPPORTED;
  GridImpl *og = m.grids[desc.out_grid];
  if (og->pub.num_dims != 3 || og->type != desc.accum_type) return PSB_ERR_UNSUPPORTED;
  return desc.accum_type == PS_FLOAT ? gt_launch<float>(m, desc, p, s, launches)
                                     : gt_launch<double>(m, desc, p, s, launches);
}

void generic_note_impl(int impl) { g_last_generic_impl = impl; }

}  // namespace psb

extern "C" psb_status psb_generic_last_impl(int *impl) {
  if (!impl) return psb::set_status(PSB_ERR_INVALID);
  *impl = psb::g_last_generic_impl;
  return PSB_OK;
}
