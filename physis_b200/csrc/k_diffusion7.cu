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

#include "device.cuh"

namespace psb {

template <typename T>
struct C7 {
  T ce, cw, cn, cs, ct, cb, cc;
};

template <typename T>
__device__ __forceinline__ T diff7_point(const C7<T> &k, T c, T w, T e, T n, T s, T b, T t) {
  T v = xmul(k.cc, c);
  v = xadd(v, xmul(k.cw, w));
  v = xadd(v, xmul(k.ce, e));
  v = xadd(v, xmul(k.cs, s));
  v = xadd(v, xmul(k.cn, n));
  v = xadd(v, xmul(k.cb, b));
  v = xadd(v, xmul(k.ct, t));
  return v;
}

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
    if (PERIODIC && images)
      store_periodic_images(o, out.sy, out.sz, out.n, out.halo, x, y, z, v);
  }
}

// --------------------------------------------------------------------------
// TMA z-streaming kernel
// --------------------------------------------------------------------------
struct TmaGeom {
  int ax0, ay0, az0;      // tensor-map coordinates of logical (0,0,0)
  int tiles_x, tiles_y;   // tiles over the domain
  int zchunk;             // planes per CTA
  int stages;             // ring depth
  int bx, by;             // box (elements)
  int stage_bytes;        // bytes between stages (128-aligned)
  int x_base;             // x of the first tile (domain lo rounded down)
};

template <typename T, bool PERIODIC>
__global__ void __launch_bounds__(512) k_diff7_tma(const __grid_constant__ CUtensorMap tin,
                                                   GridView out, int nx, int ny, int nz, Dom3 d,
                                                   C7<T> k, TmaGeom geo, int images, int *err) {
  constexpr int V = 16 / sizeof(T);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA destinations must be 128-byte aligned: align the base explicitly
  // (128 spare bytes are allocated for this).
  unsigned char *smem = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  // flags[k]: set by thread 0 before a barrier, read by all after it. The
  // two slots alternate by iteration, so a slow reader of one iteration's
  // flag never races with thread 0 writing the next one.
  volatile int *flags = reinterpret_cast<volatile int *>(smem + 8 * 32);
  unsigned char *ring = smem + 384;

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * blockDim.x + tx;
  const int TX = blockDim.x * V, TY = blockDim.y;
  const int S = geo.stages;
  int b = blockIdx.x;
  const int tile_x = b % geo.tiles_x;
  b /= geo.tiles_x;
  const int tile_y = b % geo.tiles_y;
  const int zc = b / geo.tiles_y;
  const int x0 = geo.x_base + tile_x * TX;
  const int y0 = d.lo[1] + tile_y * TY;
  const int zb = d.lo[2] + zc * geo.zchunk;
  const int ze = min(zb + geo.zchunk, d.hi[2]);
  const int nzl = ze - zb;       // output planes
  const int np = nzl + 2;        // input planes zb-1 .. ze
  const uint32_t tx_bytes = (uint32_t)(geo.bx * geo.by * sizeof(T));

  if (tid == 0) {
    for (int i = 0; i < S; i++) mbar_init(&bars[i], 1);
    flags[0] = 0;
    flags[1] = 0;
    mbar_fence_init();
    tma_prefetch_desc(&tin);
  }
  __syncthreads();
  int issued = 0;  // meaningful in thread 0 only
  auto issue = [&](int j) {
    const int slot = j % S;
    mbar_arrive_expect_tx(&bars[slot], tx_bytes);
    tma_load_3d(ring + slot * geo.stage_bytes, &tin, &bars[slot], x0 - V + geo.ax0,
                y0 - 1 + geo.ay0, zb - 1 + j + geo.az0);
  };
  if (tid == 0) {
    const int first = min(S, np);
    for (int j = 0; j < first; j++) issue(j);
    issued = first;
  }

  // Shared-memory offsets of this thread's 16-byte column in a plane.
  const int BX = geo.bx;
  const int row_c = (ty + 1) * BX + V + tx * V;
  const int row_n = row_c - BX;
  const int row_s = row_c + BX;
  auto plane = [&](int j) -> const T * {
    return reinterpret_cast<const T *>(ring + (j % S) * geo.stage_bytes);
  };

  // Prologue: planes 0 (z-1) and 1 (z). Uses flag slot 1.
  if (tid == 0) {
    bool ok = mbar_wait_bounded(&bars[0], 0) && mbar_wait_bounded(&bars[1 % S], (1 / S) & 1);
    flags[1] = ok ? 0 : 1;
  }
  __syncthreads();
  bool bad = flags[1] != 0;
  const int xg0 = x0 + tx * V;  // global x of element 0
  const int yg = y0 + ty;
  Vec16<T> vb, vc;
  if (!bad) {
    vb = lds16(plane(0) + row_c);
    vc = lds16(plane(1) + row_c);
  }
  T *o = (T *)out.origin;
  const bool row_in = yg >= d.lo[1] && yg < d.hi[1];
  for (int jj = 0; jj < nzl && !bad; jj++) {
    const int jt = jj + 2;  // plane of z+1
    if (tid == 0) flags[jj & 1] = mbar_wait_bounded(&bars[jt % S], (jt / S) & 1) ? 0 : 1;
    __syncthreads();
    if (flags[jj & 1]) {
      bad = true;
      break;
    }
    // Plane jj is no longer read by anyone: refill its slot.
    if (tid == 0 && issued < np && issued == jj + S) {
      issue(issued);
      issued++;
    }
    const T *pz = plane(jj + 1);
    const T *pt = plane(jt);
    Vec16<T> vt = lds16(pt + row_c);
    Vec16<T> vn = lds16(pz + row_n);
    Vec16<T> vs = lds16(pz + row_s);
    const T wl = pz[row_c - 1];
    const T er = pz[row_c + V];
    const int z = zb + jj;
    Vec16<T> r;
#pragma unroll
    for (int v = 0; v < V; v++) {
      const int x = xg0 + v;
      T c = vc.v[v];
      T w = v == 0 ? wl : vc.v[v - 1];
      T e = v == V - 1 ? er : vc.v[v + 1];
      T n = vn.v[v], s = vs.v[v], bb = vb.v[v], t = vt.v[v];
      if (!PERIODIC) {
        if (x == 0) w = c;
        if (x == nx - 1) e = c;
        if (yg == 0) n = c;
        if (yg == ny - 1) s = c;
        if (z == 0) bb = c;
        if (z == nz - 1) t = c;
      }
      r.v[v] = diff7_point(k, c, w, e, n, s, bb, t);
    }
    if (row_in) {
      T *dst = o + (int64_t)xg0 + (int64_t)yg * out.sy + (int64_t)z * out.sz;
      if (xg0 >= d.lo[0] && xg0 + V <= d.hi[0]) {
        stg16(dst, r);
      } else {
#pragma unroll
        for (int v = 0; v < V; v++)
          if (xg0 + v >= d.lo[0] && xg0 + v < d.hi[0]) dst[v] = r.v[v];
      }
      if (PERIODIC && images) {
#pragma unroll
        for (int v = 0; v < V; v++)
          if (xg0 + v >= d.lo[0] && xg0 + v < d.hi[0])
            store_periodic_images(o, out.sy, out.sz, out.n, out.halo, xg0 + v, yg, z, r.v[v]);
      }
    }
    vb = vc;
    vc = vt;
  }
  if (bad && tid == 0) {
    // A bounded wait gave up: record it and let the copies still in flight
    // land (bounded again) so no TMA writes into shared memory after the
    // CTA has left. The other threads simply return.
    atomicExch(err, 1);
    for (int j = 0; j < issued; j++) {
      long long t0 = clock64();
      while (!mbar_try_wait(&bars[j % S], (j / S) & 1) && clock64() - t0 < 100000000LL) {
      }
    }
  }
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

template <typename T, bool PERIODIC>
static psb_status launch_tma(MapImpl &m, const psb_tune_config &cfg, cudaStream_t s,
                             int64_t *launches) {
  constexpr int V = 16 / sizeof(T);
  GridImpl *gi = m.grids[0], *go = m.grids[1];
  Dom3 d = dom3_of(m);
  if (d.hi[0] <= d.lo[0] || d.hi[1] <= d.lo[1] || d.hi[2] <= d.lo[2]) return PSB_OK;
  int TX = std::max(V, cfg.tile_x / V * V);
  int TY = std::max(1, cfg.tile_y);
  if ((TX / V) * TY > 512) TY = 512 / (TX / V);
  TmaGeom geo;
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
  size_t smem = 128 + 384 + (size_t)geo.stages * geo.stage_bytes;
  if (smem > rt().smem_optin) return set_status(PSB_ERR_INVALID);
  auto kern = k_diff7_tma<T, PERIODIC>;
  static size_t configured[2] = {0, 0};
  size_t &conf = configured[sizeof(T) == 8];
  if (smem > 48 * 1024 && smem > conf) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)rt().smem_optin);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute");
    conf = rt().smem_optin;
  }
  int64_t nblocks = (int64_t)geo.tiles_x * geo.tiles_y * nzc;
  if (nblocks > 0x7fffffff) return set_status(PSB_ERR_INVALID);
  int images = PERIODIC && go->layout == PSB_LAYOUT_PITCHED;
  dim3 block(TX / V, TY, 1);
  kern<<<(unsigned)nblocks, block, smem, s>>>(*map, go->view(), gi->pub.dim[0], gi->pub.dim[1],
                                              gi->pub.dim[2], d, coef_from<T>(m), geo, images,
                                              rt().d_error);
  (*launches)++;
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
    psb_status st = dbl ? (periodic ? launch_tma<double, true>(m, cfg, s, launches)
                                    : launch_tma<double, false>(m, cfg, s, launches))
                        : (periodic ? launch_tma<float, true>(m, cfg, s, launches)
                                    : launch_tma<float, false>(m, cfg, s, launches));
    if (st != PSB_ERR_UNSUPPORTED) return st;
  }
  return dbl ? (periodic ? launch_plain<double, true>(m, s, launches)
                         : launch_plain<double, false>(m, s, launches))
             : (periodic ? launch_plain<float, true>(m, s, launches)
                         : launch_plain<float, false>(m, s, launches));
}

}  // namespace psb
