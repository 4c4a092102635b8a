// Batching: many independent grids of uneven sizes advanced together.
//
// A batch member is one double-buffered solve (a 7-point diffusion, clamped
// or periodic, or a Himeno Jacobi relaxation, float) of `steps` steps, i.e.
// what PSStencilRun(m(g0->g1), m(g1->g0), steps/2) does for one grid. The
// work of all members is cut into items -- (member, step, tile) where a tile
// is a 32-, 64- or 128-wide column of the member's domain (the shape that
// fits its extent best) over a z chunk -- and laid out in
// one device-side work list ordered by step, then member, then tile.
//
// Mode 0 (persistent): one launch with one CTA per resident slot. CTAs take
// items from the list with an atomic cursor; an item of step s of member m
// waits until every tile of step s-1 of m is complete (a per-member counter,
// acquire load, bounded wait). Because the list is ordered by step, every
// dependency of an item is taken by a CTA before the item itself, so the
// earliest unfinished item can always run: the launch needs no co-residency
// guarantee and cannot deadlock. Small members no longer leave the GPU idle
// between their steps and there are no launch gaps.
// Mode 1 (graph): one launch per step over all members still running, the
// sequence captured once in a CUDA graph and replayed.
// Mode 2 / 3: the per-grid loop -- each member alone, one launch per step,
// with the plain kernel (the reference's shape) or the tuned TMA kernel.
//
// Each item runs the same tile functions as the single-grid kernels (TMA
// plane ring, warp-specialised), so every member's result is bit-identical to
// running it alone. Members may also measure a convergence residual every
// `check_every` steps (7-point: |u_{n+1}-u_n|^2 and |u_{n+1}|^2; Himeno: the
// sum of ss^2) and stop early: tiles write FP64 partials, and the CTA that
// completes the last tile of a step combines them in tile order, decides, and
// only then releases the member's next step, so the decision is deterministic.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>
#include <vector>

#include "batch.h"
#include "k_diffusion7.cuh"
#include "k_himeno.cuh"

namespace psb {

// Batched items run 128 consumer threads (tile shape per member) and one
// producer warp.
constexpr int kBConsumers = 128;
constexpr int kBThreads = kBConsumers + 32;
constexpr int kBStages = 6;

struct BMember {
  int kind;
  int n[3];
  int tiles_x, tiles_y, nzc, ntiles;
  int steps;        // steps in this launch
  int step0;        // member's global step index at local step 0
  int check_every;  // 0: no checks
  double tol2;      // squared relative tolerance
  const CUtensorMap *tmap[2];
  GridView buf[2];
  Dom3 dom;
  C7<float> k7;
  float omega;
  HimenoCoef cf;
  int64_t sy, sz;
  TmaGeom dg;
  HimenoGeom hg;
  double *partials;  // [2][ntiles][2]
  unsigned *done;    // (ntiles + 1) units per step
  int *stop;         // local steps completed when converged, or -1
  double *res;       // [0] a or gosa, [1] b, [2] gosa of the first check, [3] check count
};

struct BatchDev {
  int nmembers;
  const BMember *members;
  const int *order;             // member ids sorted by steps (descending)
  const int64_t *tile_prefix;   // prefix of ntiles over `order`
  const int64_t *step_offset;   // prefix of items over steps
  int max_steps;
  int64_t total_items;
  unsigned long long *cursor;
  int *err;
};

__device__ __forceinline__ int upper_index(const int64_t *a, int n, int64_t v) {
  // largest i in [0, n) with a[i] <= v (a non-decreasing, a[0] = 0)
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (a[mid] <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_acquire_int(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Sum of two doubles per thread over the CTA in a fixed order (thread 0).
__device__ void cta_sum2(double a, double b, double *scr, double *oa, double *ob) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) {
    scr[2 * warp] = a;
    scr[2 * warp + 1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0, sb = 0;
    for (int w = 0; w < nw; w++) {
      sa += scr[2 * w];
      sb += scr[2 * w + 1];
    }
    *oa = sa;
    *ob = sb;
  }
}

// One item: tile t of local step s of member m. All threads of the CTA call
// it. Returns false if a bounded wait gave up.
template <int GROUP>
__device__ __forceinline__ bool batch_item(const BMember &M, int s, int t, unsigned char *smem,
                                           int *err) {
  const int par = (M.step0 + s) & 1;
  const int gstep = M.step0 + s;
  const bool check = M.check_every > 0 &&
                     ((gstep + 1) % M.check_every == 0 || (M.kind == BK_HIMENO && gstep == 0));
  __shared__ int skip_s;
  if (threadIdx.x == 0) {
    const int st = ld_acquire_int(M.stop);
    skip_s = st >= 0 && s >= st;
  }
  __syncthreads();
  const bool skip = skip_s;
  int tt = t;
  const int tile_x = tt % M.tiles_x;
  tt /= M.tiles_x;
  const int tile_y = tt % M.tiles_y;
  const int zc = tt / M.tiles_y;
  double a = 0, b = 0;
  bool bad = false;
  if (!skip) {
    if (threadIdx.x == kBConsumers)  // producer: order generic acquire before TMA reads
      asm volatile("fence.proxy.async.global;" ::: "memory");
    if constexpr (GROUP == 1) {
      double g = 0;
      himeno_tile(M.tmap[par], (float *)M.buf[par ^ 1].origin, M.cf, M.sy, M.sz, M.dom, M.omega,
                  M.hg, tile_x, tile_y, zc, err, smem, &g, &bad);
      a = g;
    } else {
      TileAcc acc{0, 0};
      const int images = M.kind == BK_DIFF7P;
      if (M.kind == BK_DIFF7P) {
        if (check)
          diff7_tile<float, true, true>(M.tmap[par], M.buf[par ^ 1], M.n[0], M.n[1], M.n[2], M.dom,
                                        M.k7, M.dg, tile_x, tile_y, zc, images, err, smem, &acc);
        else
          diff7_tile<float, true, false>(M.tmap[par], M.buf[par ^ 1], M.n[0], M.n[1], M.n[2],
                                         M.dom, M.k7, M.dg, tile_x, tile_y, zc, images, err, smem,
                                         nullptr);
      } else {
        if (check)
          diff7_tile<float, false, true>(M.tmap[par], M.buf[par ^ 1], M.n[0], M.n[1], M.n[2],
                                         M.dom, M.k7, M.dg, tile_x, tile_y, zc, 0, err, smem,
                                         &acc);
        else
          diff7_tile<float, false, false>(M.tmap[par], M.buf[par ^ 1], M.n[0], M.n[1], M.n[2],
                                          M.dom, M.k7, M.dg, tile_x, tile_y, zc, 0, err, smem,
                                          nullptr);
      }
      a = acc.a;
      b = acc.b;
    }
  }
  // Every thread is past the tile (the ring is idle): reuse the ring area.
  double *scr = reinterpret_cast<double *>(smem + 512);
  if (check && !skip) {
    double sa, sb;
    cta_sum2(a, b, scr, &sa, &sb);
    if (threadIdx.x == 0) {
      M.partials[(par * M.ntiles + t) * 2] = sa;
      M.partials[(par * M.ntiles + t) * 2 + 1] = sb;
    }
  }
  __shared__ int bad_any;
  if (threadIdx.x == 0) bad_any = 0;
  __syncthreads();
  if (bad) atomicExch(&bad_any, 1);
  __syncthreads();
  if (threadIdx.x == 0 && !bad_any) {
    __threadfence();
    const unsigned unit = (unsigned)M.ntiles + 1;
    const unsigned old = atomicAdd(M.done, 1u);
    if (old + 1 == (unsigned)s * unit + (unsigned)M.ntiles) {
      // Last tile of this step: decide convergence, then release the step.
      if (check && !skip) {
        __threadfence();
        double sa = 0, sb = 0;
        for (int i = 0; i < M.ntiles; i++) {
          sa += __ldcg(&M.partials[(par * M.ntiles + i) * 2]);
          sb += __ldcg(&M.partials[(par * M.ntiles + i) * 2 + 1]);
        }
        bool conv;
        if (M.kind == BK_HIMENO) {
          if (gstep == 0) M.res[2] = sa;
          const double g0 = gstep == 0 ? sa : __ldcg(&M.res[2]);
          conv = sa <= M.tol2 * g0;
          M.res[1] = g0;
        } else {
          conv = sa <= M.tol2 * sb;
          M.res[1] = sb;
        }
        M.res[0] = sa;
        M.res[3] = (double)(gstep + 1);
        if (conv && M.tol2 > 0) atomicExch(M.stop, s + 1);
      }
      __threadfence();
      atomicAdd(M.done, 1u);
    }
  }
  return !bad_any;
}

__device__ __forceinline__ unsigned char *aligned_smem(unsigned char *raw) {
  return raw + ((128 - (smem_u32(raw) & 127)) & 127);
}

// Retire the ring's barriers between items (they are initialised again by
// the next tile).
__device__ __forceinline__ void inval_barriers(unsigned char *smem) {
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  for (int i = 0; i < kBStages; i++) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&full[i])) : "memory");
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(&full[32 + i])) : "memory");
  }
}

// Mode 0: one persistent launch per stencil kind over that kind's work list
// (a kernel per kind keeps each at the register budget of its single-grid
// kernel; the two lists are independent).
// Diffusion items (four instantiations of the tile: clamped/periodic, with or
// without residual terms) get the register budget of 3 CTAs per SM, Himeno
// items that of 4.
template <int GROUP>
__global__ void __launch_bounds__(kBThreads, GROUP == 0 ? 3 : 4) k_batch_persistent(BatchDev B) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = aligned_smem(smem_raw);
  __shared__ long long item_s;
  __shared__ int m_s, s_s, t_s, stop_s;
  if (threadIdx.x == 0) stop_s = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      const long long item = (long long)atomicAdd(B.cursor, 1ull);
      item_s = item;
      if (item < B.total_items) {
        const int s = upper_index(B.step_offset, B.max_steps + 1, item);
        const int64_t local = item - B.step_offset[s];
        const int k = upper_index(B.tile_prefix, B.nmembers + 1, local);
        const int m = B.order[k];
        m_s = m;
        s_s = s;
        t_s = (int)(local - B.tile_prefix[k]);
        // Wait for every tile of step s-1 of this member (bounded).
        const BMember &M = B.members[m];
        const unsigned need = (unsigned)s * ((unsigned)M.ntiles + 1);
        if (ld_acquire(M.done) < need) {
          long long t0 = clock64();
          unsigned sleep = 32;
          while (ld_acquire(M.done) < need) {
            if (ld_acquire_int((const int *)B.err) != 0 || clock64() - t0 > 4000000000LL) {
              atomicExch(B.err, 1);
              stop_s = 1;
              break;
            }
            __nanosleep(sleep);
            if (sleep < 2048) sleep <<= 1;
          }
        }
      }
    }
    __syncthreads();
    if (item_s >= B.total_items || stop_s) break;
    if (!batch_item<GROUP>(B.members[m_s], s_s, t_s, smem, B.err)) {
      __syncthreads();
      break;
    }
    __syncthreads();
    if (threadIdx.x == 0) inval_barriers(smem);
    __syncthreads();
  }
}

// Mode 1: one launch per step and kind; blockIdx.x enumerates the tiles of
// that kind's members still running at step s.
template <int GROUP>
__global__ void __launch_bounds__(kBThreads, GROUP == 0 ? 3 : 4) k_batch_step(BatchDev B, int s) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *smem = aligned_smem(smem_raw);
  const int64_t local = blockIdx.x;
  const int k = upper_index(B.tile_prefix, B.nmembers + 1, local);
  const int m = B.order[k];
  const int t = (int)(local - B.tile_prefix[k]);
  batch_item<GROUP>(B.members[m], s, t, smem, B.err);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

}  // namespace psb

using namespace psb;

// Work list of one kernel kind (group 0: diffusion members, 1: Himeno).
struct BatchGroup {
  std::vector<int> order;               // member ids of this group, by steps (descending)
  std::vector<int64_t> tile_prefix, step_offset;
  int max_steps = 0;
  int64_t total_items = 0;
  int *d_order = nullptr;
  int64_t *d_tile_prefix = nullptr;
  int64_t *d_step_offset = nullptr;
  unsigned long long *d_cursor = nullptr;
  size_t cap_order = 0, cap_tile_prefix = 0, cap_step_offset = 0;
  int blocks_persistent = 0;
};

struct psb_batch {
  std::vector<BatchMemberHost> hm;
  std::vector<double> res_init;  // 4 per member, uploaded by batch_prepare when set
  BMember *d_members = nullptr;
  CUtensorMap *d_tmaps = nullptr;
  double *d_partials = nullptr;
  unsigned *d_done = nullptr;
  int *d_stop = nullptr;
  double *d_res = nullptr;
  size_t cap_members = 0, cap_tmaps = 0, cap_partials = 0, cap_done = 0, cap_stop = 0,
         cap_res = 0;  // bytes allocated (device buffers are reused while they fit)
  std::vector<BMember> members;
  BatchGroup grp[2];
  bool built = false;
  cudaGraphExec_t graph = nullptr;
  cudaStream_t side = nullptr;       // second stream of the per-step graph
  cudaEvent_t fork = nullptr, join = nullptr;
  double last_ms = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // batch timing (apart from PSStencilRun's)
  int64_t last_launches = 0;
  int64_t last_lups = 0;
};

namespace psb {

static int member_group(int kind) { return kind == BK_HIMENO ? 1 : 0; }

// The work lists and descriptors no longer match the members.
static void batch_invalidate(psb_batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->built = false;
}

static void batch_release_device(psb_batch *b) {
  batch_invalidate(b);
  cudaFree(b->d_members);
  cudaFree(b->d_tmaps);
  cudaFree(b->d_partials);
  cudaFree(b->d_done);
  cudaFree(b->d_stop);
  cudaFree(b->d_res);
  b->d_members = nullptr;
  b->d_tmaps = nullptr;
  b->d_partials = nullptr;
  b->d_done = nullptr;
  b->d_stop = nullptr;
  b->d_res = nullptr;
  b->cap_members = b->cap_tmaps = b->cap_partials = b->cap_done = b->cap_stop = b->cap_res = 0;
  for (auto &g : b->grp) {
    cudaFree(g.d_order);
    cudaFree(g.d_tile_prefix);
    cudaFree(g.d_step_offset);
    cudaFree(g.d_cursor);
    g = BatchGroup();
  }
}

// Make *p hold at least `bytes` (grown by half again when it must grow, so
// a server's changing member list rarely reallocates).
template <typename T>
static psb_status dev_reserve(T **p, size_t *cap, size_t bytes) {
  bytes = std::max<size_t>(bytes, 16);
  if (bytes <= *cap) return PSB_OK;
  const size_t want = std::max(bytes, *cap + *cap / 2);
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  PSB_TRY(cudaMalloc((void **)p, want));
  *cap = want;
  return PSB_OK;
}

// Tile shapes of batched items: 128 consumer threads as 8 x 16, 16 x 8 or
// 32 x 4 (x threads of 4 floats each x rows); each member takes the shape
// with the fewest tiles over its x-y extent (then the fewest box elements),
// so small and narrow members waste few threads on partial tiles.
constexpr int kBShapes[3][2] = {{8, 16}, {16, 8}, {32, 4}};

static void pick_shape(int nx, int ny, int rows_per_thread, int *tx_threads, int *ty_threads) {
  int64_t best_tiles = -1, best_box = 0;
  for (const auto &sh : kBShapes) {
    const int TX = sh[0] * 4, TY = sh[1] * rows_per_thread;
    const int64_t tiles = (int64_t)((nx + TX - 1) / TX) * ((ny + TY - 1) / TY);
    const int64_t box = tiles * (TX + 8) * (TY + 2);
    if (best_tiles < 0 || tiles < best_tiles || (tiles == best_tiles && box < best_box)) {
      best_tiles = tiles;
      best_box = box;
      *tx_threads = sh[0];
      *ty_threads = sh[1];
    }
  }
}

static int stage_bytes_of(int tx_threads, int ty_threads, int rows_per_thread) {
  return ((tx_threads * 4 + 8) * (ty_threads * rows_per_thread + 2) * 4 + 127) / 128 * 128;
}

static TmaGeom batch_dgeom(const GridImpl *g) {
  TmaGeom geo;
  pick_shape(g->pub.dim[0], g->pub.dim[1], kVY, &geo.tx_threads, &geo.ty_threads);
  const int TX = geo.tx_threads * 4, TY = geo.ty_threads * kVY;
  geo.bx = TX + 8;
  geo.by = TY + 2;
  geo.ax0 = g->pad_left;
  geo.ay0 = g->halo;
  geo.az0 = g->halo;
  geo.x_base = 0;
  geo.tiles_x = (g->pub.dim[0] + TX - 1) / TX;
  geo.tiles_y = (g->pub.dim[1] + TY - 1) / TY;
  geo.zchunk = 64;
  geo.stages = kBStages;
  geo.stage_bytes = stage_bytes_of(geo.tx_threads, geo.ty_threads, kVY);
  return geo;
}

static HimenoGeom batch_hgeom(const GridImpl *g) {
  HimenoGeom geo;
  // interior domain [1, n-1): tiles start at x = 0 (x_base), y = 1.
  pick_shape(g->pub.dim[0] - 1, g->pub.dim[1] - 2, 1, &geo.tx_threads, &geo.ty_threads);
  const int TX = geo.tx_threads * 4, TY = geo.ty_threads;
  geo.bx = TX + 8;
  geo.by = TY + 2;
  geo.ax0 = g->pad_left;
  geo.ay0 = g->halo;
  geo.az0 = g->halo;
  geo.x_base = 0;
  geo.tiles_x = (g->pub.dim[0] - 1 + TX - 1) / TX;
  geo.tiles_y = (g->pub.dim[1] - 2 + TY - 1) / TY;
  geo.zchunk = 64;
  geo.stages = kBStages;
  geo.stage_bytes = stage_bytes_of(geo.tx_threads, geo.ty_threads, 1);
  geo.nx = g->pub.dim[0];
  return geo;
}

static size_t batch_smem(int group) {
  int stage = 0;
  for (const auto &sh : kBShapes)
    stage = std::max(stage, stage_bytes_of(sh[0], sh[1], group == 0 ? kVY : 1));
  return group == 0 ? 128 + 512 + (size_t)kBStages * stage : 128 + 768 + (size_t)kBStages * stage;
}

// Build the device work lists and member descriptors for one launch in which
// member i runs steps[i] steps starting at its global step step0[i].
psb_status batch_prepare(psb_batch *b, const std::vector<int> &steps, const std::vector<int> &step0) {
  Runtime &r = rt();
  const int n = (int)b->hm.size();
  batch_invalidate(b);
  b->members.assign(n, BMember());
  std::vector<CUtensorMap> tmaps(2 * std::max(1, n));
  int64_t partial_slots = 0;
  for (int i = 0; i < n; i++) {
    const BatchMemberHost &h = b->hm[i];
    BMember &M = b->members[i];
    memset(&M, 0, sizeof(M));
    M.kind = h.kind;
    GridImpl *g0 = h.grids[0], *g1 = h.grids[1];
    for (int k = 0; k < 3; k++) M.n[k] = g0->pub.dim[k];
    M.steps = steps[i];
    M.step0 = step0[i];
    M.check_every = h.check_every;
    M.tol2 = h.tol * h.tol;
    M.buf[0] = g0->view();
    M.buf[1] = g1->view();
    M.sy = g0->sy;
    M.sz = g0->sz;
    const CUtensorMap *a = nullptr, *c = nullptr;
    if (h.kind == BK_HIMENO) {
      M.hg = batch_hgeom(g0);
      for (int k = 0; k < 3; k++) {
        M.dom.lo[k] = 1;
        M.dom.hi[k] = g0->pub.dim[k] - 1;
      }
      M.tiles_x = M.hg.tiles_x;
      M.tiles_y = M.hg.tiles_y;
      M.nzc = (g0->pub.dim[2] - 2 + M.hg.zchunk - 1) / M.hg.zchunk;
      M.omega = (float)h.params[0];
      for (int k = 0; k < 12; k++) M.cf.f[k] = (const float *)h.grids[2 + k]->view().origin;
      PSB_CHECK(get_tmap(g0, M.hg.bx, M.hg.by, &a));
      PSB_CHECK(get_tmap(g1, M.hg.bx, M.hg.by, &c));
    } else {
      M.dg = batch_dgeom(g0);
      for (int k = 0; k < 3; k++) {
        M.dom.lo[k] = 0;
        M.dom.hi[k] = g0->pub.dim[k];
      }
      M.tiles_x = M.dg.tiles_x;
      M.tiles_y = M.dg.tiles_y;
      M.nzc = (g0->pub.dim[2] + M.dg.zchunk - 1) / M.dg.zchunk;
      M.k7.ce = (float)h.params[0];
      M.k7.cw = (float)h.params[1];
      M.k7.cn = (float)h.params[2];
      M.k7.cs = (float)h.params[3];
      M.k7.ct = (float)h.params[4];
      M.k7.cb = (float)h.params[5];
      M.k7.cc = (float)h.params[6];
      PSB_CHECK(get_tmap(g0, M.dg.bx, M.dg.by, &a));
      PSB_CHECK(get_tmap(g1, M.dg.bx, M.dg.by, &c));
    }
    tmaps[2 * i] = *a;
    tmaps[2 * i + 1] = *c;
    M.ntiles = M.tiles_x * M.tiles_y * M.nzc;
    partial_slots += 4 * (int64_t)M.ntiles;
  }
  PSB_CHECK(dev_reserve(&b->d_tmaps, &b->cap_tmaps, sizeof(CUtensorMap) * tmaps.size()));
  PSB_TRY(cudaMemcpy(b->d_tmaps, tmaps.data(), sizeof(CUtensorMap) * tmaps.size(),
                     cudaMemcpyHostToDevice));
  PSB_CHECK(dev_reserve(&b->d_partials, &b->cap_partials,
                        sizeof(double) * std::max<int64_t>(1, partial_slots)));
  PSB_CHECK(dev_reserve(&b->d_done, &b->cap_done, sizeof(unsigned) * std::max(1, n)));
  PSB_CHECK(dev_reserve(&b->d_stop, &b->cap_stop, sizeof(int) * std::max(1, n)));
  PSB_CHECK(dev_reserve(&b->d_res, &b->cap_res, sizeof(double) * 4 * std::max(1, n)));
  if ((int)b->res_init.size() == 4 * n && n > 0)
    PSB_TRY(cudaMemcpy(b->d_res, b->res_init.data(), sizeof(double) * 4 * n, cudaMemcpyHostToDevice));
  else
    PSB_TRY(cudaMemset(b->d_res, 0, sizeof(double) * 4 * std::max(1, n)));
  int64_t off = 0;
  for (int i = 0; i < n; i++) {
    BMember &M = b->members[i];
    M.tmap[0] = b->d_tmaps + 2 * i;
    M.tmap[1] = b->d_tmaps + 2 * i + 1;
    M.partials = b->d_partials + off;
    off += 4 * (int64_t)M.ntiles;
    M.done = b->d_done + i;
    M.stop = b->d_stop + i;
    M.res = b->d_res + 4 * i;
  }
  PSB_CHECK(dev_reserve(&b->d_members, &b->cap_members, sizeof(BMember) * std::max(1, n)));
  PSB_TRY(cudaMemcpy(b->d_members, b->members.data(), sizeof(BMember) * n, cudaMemcpyHostToDevice));
  // One work list per kernel kind. Members are ordered by steps
  // (descending), so the members still running at step s are a prefix.
  for (int gi = 0; gi < 2; gi++) {
    BatchGroup &G = b->grp[gi];
    G.order.clear();
    for (int i = 0; i < n; i++)
      if (member_group(b->hm[i].kind) == gi) G.order.push_back(i);
    std::stable_sort(G.order.begin(), G.order.end(),
                     [&](int x, int y) { return steps[x] > steps[y]; });
    const int gn = (int)G.order.size();
    G.tile_prefix.assign(gn + 1, 0);
    for (int i = 0; i < gn; i++)
      G.tile_prefix[i + 1] = G.tile_prefix[i] + b->members[G.order[i]].ntiles;
    G.max_steps = gn ? steps[G.order[0]] : 0;
    G.step_offset.assign(G.max_steps + 1, 0);
    int active = gn;
    for (int st = 0; st < G.max_steps; st++) {
      while (active > 0 && steps[G.order[active - 1]] <= st) active--;
      G.step_offset[st + 1] = G.step_offset[st] + G.tile_prefix[active];
    }
    G.total_items = G.max_steps ? G.step_offset[G.max_steps] : 0;
    PSB_CHECK(dev_reserve(&G.d_order, &G.cap_order, sizeof(int) * std::max(1, gn)));
    if (gn) PSB_TRY(cudaMemcpy(G.d_order, G.order.data(), sizeof(int) * gn, cudaMemcpyHostToDevice));
    PSB_CHECK(dev_reserve(&G.d_tile_prefix, &G.cap_tile_prefix, sizeof(int64_t) * (gn + 1)));
    PSB_TRY(cudaMemcpy(G.d_tile_prefix, G.tile_prefix.data(), sizeof(int64_t) * (gn + 1),
                       cudaMemcpyHostToDevice));
    PSB_CHECK(dev_reserve(&G.d_step_offset, &G.cap_step_offset,
                          sizeof(int64_t) * (G.max_steps + 1)));
    PSB_TRY(cudaMemcpy(G.d_step_offset, G.step_offset.data(), sizeof(int64_t) * (G.max_steps + 1),
                       cudaMemcpyHostToDevice));
    if (!G.d_cursor) PSB_TRY(cudaMalloc(&G.d_cursor, sizeof(unsigned long long)));
    int per_sm = 0;
    if (gi == 0) {
      PSB_TRY(cudaFuncSetAttribute(k_batch_persistent<0>,
                                   cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
      PSB_TRY(cudaFuncSetAttribute(k_batch_step<0>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
      PSB_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_persistent<0>,
                                                            kBThreads, batch_smem(0)));
    } else {
      PSB_TRY(cudaFuncSetAttribute(k_batch_persistent<1>,
                                   cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
      PSB_TRY(cudaFuncSetAttribute(k_batch_step<1>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   cudaSharedmemCarveoutMaxShared));
      PSB_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_persistent<1>,
                                                            kBThreads, batch_smem(1)));
    }
    G.blocks_persistent = std::max(1, per_sm) * r.sm_count;
  }
  b->built = true;
  return PSB_OK;
}

// After a run: per member, local steps completed when it converged (-1 if
// it did not) and its residual state (4 doubles).
psb_status batch_read_state(psb_batch *b, std::vector<int> &stop, std::vector<double> &res) {
  const int n = (int)b->hm.size();
  stop.assign(n, -1);
  res.assign(4 * n, 0.0);
  if (!b->built || n == 0) return PSB_OK;
  PSB_TRY(cudaMemcpy(stop.data(), b->d_stop, sizeof(int) * n, cudaMemcpyDeviceToHost));
  PSB_TRY(cudaMemcpy(res.data(), b->d_res, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost));
  return PSB_OK;
}

psb_status batch_reset_counters(psb_batch *b, cudaStream_t s) {
  const int n = (int)b->hm.size();
  PSB_TRY(cudaMemsetAsync(b->d_done, 0, sizeof(unsigned) * std::max(1, n), s));
  PSB_TRY(cudaMemsetAsync(b->d_stop, 0xff, sizeof(int) * std::max(1, n), s));
  for (auto &g : b->grp) PSB_TRY(cudaMemsetAsync(g.d_cursor, 0, sizeof(unsigned long long), s));
  return PSB_OK;
}

static BatchDev batch_dev(psb_batch *b, int gi) {
  const BatchGroup &G = b->grp[gi];
  BatchDev B;
  B.nmembers = (int)G.order.size();
  B.members = b->d_members;
  B.order = G.d_order;
  B.tile_prefix = G.d_tile_prefix;
  B.step_offset = G.d_step_offset;
  B.max_steps = G.max_steps;
  B.total_items = G.total_items;
  B.cursor = G.d_cursor;
  B.err = rt().d_error;
  return B;
}

psb_status batch_launch_persistent(psb_batch *b, cudaStream_t s, int64_t *launches) {
  PSB_CHECK(batch_reset_counters(b, s));
  for (int gi = 0; gi < 2; gi++) {
    const BatchGroup &G = b->grp[gi];
    if (!G.total_items) continue;
    const int blocks = (int)std::min<int64_t>(G.blocks_persistent, G.total_items);
    if (gi == 0)
      k_batch_persistent<0><<<blocks, kBThreads, batch_smem(0), s>>>(batch_dev(b, 0));
    else
      k_batch_persistent<1><<<blocks, kBThreads, batch_smem(1), s>>>(batch_dev(b, 1));
    (*launches)++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "k_batch_persistent");
  }
  return PSB_OK;
}

// Per-step launches (mode 1): both kinds' step sequences, on two streams
// forked and joined inside one CUDA graph, recorded once and replayed.
psb_status batch_launch_graph(psb_batch *b, cudaStream_t s, int64_t *launches) {
  if (!b->graph) {
    if (!b->side) {
      PSB_TRY(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
      PSB_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
      PSB_TRY(cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming));
    }
    cudaGraph_t g;
    PSB_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    psb_status st = batch_reset_counters(b, s);
    cudaEventRecord(b->fork, s);
    cudaStreamWaitEvent(b->side, b->fork, 0);
    for (int gi = 0; gi < 2 && st == PSB_OK; gi++) {
      const BatchGroup &G = b->grp[gi];
      cudaStream_t ss = gi == 0 ? s : b->side;
      const BatchDev B = batch_dev(b, gi);
      int active = (int)G.order.size();
      for (int step = 0; step < G.max_steps; step++) {
        while (active > 0 && b->members[G.order[active - 1]].steps <= step) active--;
        const unsigned blocks = (unsigned)G.tile_prefix[active];
        if (gi == 0)
          k_batch_step<0><<<blocks, kBThreads, batch_smem(0), ss>>>(B, step);
        else
          k_batch_step<1><<<blocks, kBThreads, batch_smem(1), ss>>>(B, step);
      }
    }
    cudaEventRecord(b->join, b->side);
    cudaStreamWaitEvent(s, b->join, 0);
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (st != PSB_OK || e != cudaSuccess) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      cudaGetLastError();
      return st != PSB_OK ? set_status(st) : cuda_status(e, "batch graph capture");
    }
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_status(e, "batch graph instantiate");
  }
  PSB_TRY(cudaGraphLaunch(b->graph, s));
  *launches += b->grp[0].max_steps + b->grp[1].max_steps;
  return PSB_OK;
}

}  // namespace psb

// ===========================================================================
// C ABI
// ===========================================================================
namespace psb {

psb_batch *batch_new() {
  psb_batch *b = new psb_batch();
  cudaEventCreate(&b->ev0);
  cudaEventCreate(&b->ev1);
  return b;
}

void batch_set_members(psb_batch *b, const std::vector<BatchMemberHost> &m,
                       const std::vector<double> &res_init) {
  batch_invalidate(b);
  b->hm = m;
  b->res_init = res_init;
}

void batch_delete(psb_batch *b) {
  if (!b) return;
  batch_release_device(b);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->join) cudaEventDestroy(b->join);
  delete b;
}

psb_status batch_add_member(psb_batch *b, const BatchMemberHost &m) {
  b->hm.push_back(m);
  batch_invalidate(b);
  return PSB_OK;
}

// Per-grid loop (modes 2 and 3): each member alone with one launch per step.
static psb_status batch_run_loop(psb_batch *b, int impl, int64_t *launches) {
  Runtime &r = rt();
  const int old_impl = r.impl;
  const bool old_graph = r.use_graph;
  r.impl = impl;
  r.use_graph = impl != PSB_IMPL_PLAIN;  // the plain loop launches every step itself
  drop_all_graphs();
  psb_status st = PSB_OK;
  for (auto &h : b->hm) {
    __PSDomain dom = h.kind == BK_HIMENO
                         ? PSDomain3DNew(1, h.grids[0]->pub.dim[0] - 1, 1, h.grids[0]->pub.dim[1] - 1,
                                         1, h.grids[0]->pub.dim[2] - 1)
                         : PSDomain3DNew(0, h.grids[0]->pub.dim[0], 0, h.grids[0]->pub.dim[1], 0,
                                         h.grids[0]->pub.dim[2]);
    __PSGrid *fw[14], *bw[14];
    for (int i = 0; i < h.ngrids; i++) fw[i] = bw[i] = &h.grids[i]->pub;
    bw[0] = &h.grids[1]->pub;
    bw[1] = &h.grids[0]->pub;
    PSStencil m1 = 0, m2 = 0;
    st = psb_stencil_map(h.kernel_id, &dom, fw, h.ngrids, h.params, h.nparams, &m1);
    if (st == PSB_OK) st = psb_stencil_map(h.kernel_id, &dom, bw, h.ngrids, h.params, h.nparams, &m2);
    if (st == PSB_OK) {
      PSStencil ms[2] = {m1, m2};
      if (h.steps / 2) {
        st = psb_stencil_run(ms, 2, h.steps / 2);
        *launches += r.last_launches;
      }
      if (st == PSB_OK && (h.steps & 1)) {
        st = psb_stencil_run(ms, 1, 1);
        *launches += r.last_launches;
      }
    }
    if (m1) psb_stencil_free(m1);
    if (m2) psb_stencil_free(m2);
    if (st != PSB_OK) break;
  }
  r.impl = old_impl;
  r.use_graph = old_graph;
  drop_all_graphs();
  return st;
}

}  // namespace psb

extern "C" {

psb_status psb_batch_create(psb_batch **b) {
  if (!b) return set_status(PSB_ERR_INVALID);
  PSB_CHECK(ensure_init());
  *b = new psb_batch();
  PSB_TRY(cudaEventCreate(&(*b)->ev0));
  PSB_TRY(cudaEventCreate(&(*b)->ev1));
  return PSB_OK;
}

psb_status psb_batch_add(psb_batch *b, int kernel_id, __PSGrid *const *grids, int ngrids,
                         const double *params, int nparams, int steps, int *member) {
  if (!b || !grids || steps < 0 || nparams < 0 || nparams > PSB_MAX_PARAMS)
    return set_status(PSB_ERR_INVALID);
  BatchMemberHost h;
  h.kernel_id = kernel_id;
  if (kernel_id == PSB_KERNEL_DIFFUSION7 || kernel_id == PSB_KERNEL_DIFFUSION7_PERIODIC) {
    if (ngrids != 2 || nparams != 7) return set_status(PSB_ERR_INVALID);
    h.kind = kernel_id == PSB_KERNEL_DIFFUSION7 ? BK_DIFF7 : BK_DIFF7P;
  } else if (kernel_id == PSB_KERNEL_HIMENO19) {
    if (ngrids != 14 || nparams != 1) return set_status(PSB_ERR_INVALID);
    h.kind = BK_HIMENO;
  } else {
    return set_status(PSB_ERR_UNSUPPORTED);
  }
  h.ngrids = ngrids;
  for (int i = 0; i < ngrids; i++) {
    GridImpl *g = as_impl(grids[i]);
    if (!g || g->layout != PSB_LAYOUT_PITCHED || g->type != PS_FLOAT || g->pub.num_dims != 3)
      return set_status(PSB_ERR_INVALID);
    for (int k = 0; k < 3; k++)
      if (g->pub.dim[k] != as_impl(grids[0])->pub.dim[k]) return set_status(PSB_ERR_INVALID);
    h.grids[i] = g;
  }
  if (h.grids[0] == h.grids[1]) return set_status(PSB_ERR_INVALID);
  const int *n = h.grids[0]->pub.dim;
  if (h.kind == BK_HIMENO && (n[0] < 3 || n[1] < 3 || n[2] < 3)) return set_status(PSB_ERR_INVALID);
  if (h.kind == BK_DIFF7P && (n[0] < PSB_HALO || n[1] < PSB_HALO || n[2] < PSB_HALO))
    return set_status(PSB_ERR_INVALID);
  for (int i = 0; i < nparams; i++) h.params[i] = params[i];
  h.nparams = nparams;
  h.steps = steps;
  h.points = h.kind == BK_HIMENO ? (int64_t)(n[0] - 2) * (n[1] - 2) * (n[2] - 2)
                                 : (int64_t)n[0] * n[1] * n[2];
  if (member) *member = (int)b->hm.size();
  return batch_add_member(b, h);
}

psb_status psb_batch_run(psb_batch *b, int mode) {
  if (!b) return set_status(PSB_ERR_INVALID);
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  int64_t launches = 0;
  legacy_join_in();
  // Periodic members read their input's resident halo.
  for (auto &h : b->hm)
    if (h.kind == BK_DIFF7P && h.grids[0]->ghost_valid != PSB_BOUNDARY_PERIODIC)
      PSB_CHECK(launch_halo_fill(h.grids[0], PSB_BOUNDARY_PERIODIC, r.stream));
  if (mode == 0 || mode == 1) {
    if (!b->built) {
      std::vector<int> steps, step0;
      for (auto &h : b->hm) {
        steps.push_back(h.steps);
        step0.push_back(0);
      }
      PSB_CHECK(batch_prepare(b, steps, step0));
    }
  }
  PSB_TRY(cudaEventRecord(b->ev0, r.stream));
  psb_status st;
  switch (mode) {
    case 0: st = batch_launch_persistent(b, r.stream, &launches); break;
    case 1: st = batch_launch_graph(b, r.stream, &launches); break;
    case 2: st = batch_run_loop(b, PSB_IMPL_PLAIN, &launches); break;
    case 3: st = batch_run_loop(b, PSB_IMPL_AUTO, &launches); break;
    default: return set_status(PSB_ERR_INVALID);
  }
  if (st != PSB_OK) return set_status(st);
  PSB_TRY(cudaEventRecord(b->ev1, r.stream));
  legacy_join_out();
  PSB_TRY(cudaEventSynchronize(b->ev1));
  float ms = 0;
  PSB_TRY(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  b->last_ms = ms;
  b->last_launches = launches;
  int64_t lups = 0;
  for (auto &h : b->hm) {
    lups += h.points * h.steps;
    // Writers keep the output halo of periodic members current.
    if (h.kind == BK_DIFF7P) {
      h.grids[0]->ghost_valid = PSB_BOUNDARY_PERIODIC;
      h.grids[1]->ghost_valid = PSB_BOUNDARY_PERIODIC;
    } else {
      h.grids[0]->ghost_valid = h.grids[1]->ghost_valid = PSB_BOUNDARY_NONE;
    }
  }
  b->last_lups = lups;
  int err = 0;
  PSB_TRY(cudaMemcpy(&err, r.d_error, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(r.d_error, 0, sizeof(int));
    return set_status(PSB_ERR_TIMEOUT);
  }
  return PSB_OK;
}

psb_status psb_batch_stats(psb_batch *b, double *device_ms, int64_t *launches,
                           int64_t *lattice_updates) {
  if (!b) return set_status(PSB_ERR_INVALID);
  if (device_ms) *device_ms = b->last_ms;
  if (launches) *launches = b->last_launches;
  if (lattice_updates) *lattice_updates = b->last_lups;
  return PSB_OK;
}

psb_status psb_batch_set_stop(psb_batch *b, int member, double tol, int check_every) {
  if (!b || member < 0 || member >= (int)b->hm.size() || tol < 0 || check_every < 0)
    return set_status(PSB_ERR_INVALID);
  b->hm[member].tol = tol;
  b->hm[member].check_every = check_every;
  batch_invalidate(b);
  return PSB_OK;
}

psb_status psb_batch_member_result(psb_batch *b, int member, int *steps_done, double *residual,
                                   int *result_grid) {
  if (!b || member < 0 || member >= (int)b->hm.size()) return set_status(PSB_ERR_INVALID);
  const BatchMemberHost &h = b->hm[member];
  int done = h.steps;
  double res = -1.0;
  if (b->built) {
    int stop = -1;
    double r4[4];
    PSB_TRY(cudaMemcpy(&stop, b->d_stop + member, sizeof(int), cudaMemcpyDeviceToHost));
    PSB_TRY(cudaMemcpy(r4, b->d_res + 4 * member, sizeof(r4), cudaMemcpyDeviceToHost));
    if (stop >= 0) done = stop;
    if (r4[3] > 0) res = r4[1] > 0 ? sqrt(r4[0] / r4[1]) : 0.0;
  }
  if (steps_done) *steps_done = done;
  if (residual) *residual = res;
  if (result_grid) *result_grid = done & 1;
  return PSB_OK;
}

psb_status psb_batch_free(psb_batch *b) {
  if (!b) return set_status(PSB_ERR_INVALID);
  cudaStreamSynchronize(rt().stream);
  batch_release_device(b);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->join) cudaEventDestroy(b->join);
  delete b;
  return PSB_OK;
}

}  // extern "C"
