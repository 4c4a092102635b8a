// Generic flat linear stencil and halo maintenance.
//
// k_generic applies a registered psb_generic_stencil: out(p) = post(p) *
// (t0 + t1 + ... ) with ti = a_i * b_i, each factor a grid read at p + offset
// (with the per-access index forms of the reference: plain, periodic
// (i+n)%n as in include/physis/physis_cuda.h:208-231, or clamped) or a
// constant, converted to the accumulation type and summed left to right. It
// is the executable form of the user stencils in the reference's system
// tests (tests/system_tests/test_cases/test_*.c) that are flat sums of
// products, including grids of lower dimension read inside a 3-D stencil
// (test_mixed-dim*.c), mixed element types (test_7-pt-type-mix.c) and
// red-black ordering (test_redblack*.c).
//
// k_halo_fill rewrites the resident halo of a pitched grid so that ghost
// cell q holds the periodic image of the interior (used once, before the
// first periodic TMA read of a grid whose halo is stale).
#include <algorithm>

#include "k_generic.cuh"
#include "reduce.cuh"

namespace psb {

template <typename A>
__global__ void __launch_bounds__(256) k_generic(const GenTable *__restrict__ tab, GenGrids G,
                                                 Dom3 d, int color) {
  __shared__ GenTable t;
  // Stage the term table in shared memory (a few KB, read by every point).
  {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nt = blockDim.x * blockDim.y * blockDim.z;
    const int words = sizeof(GenTable) / 4;
    const uint32_t *src = reinterpret_cast<const uint32_t *>(tab);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&t);
    for (int i = tid; i < words; i += nt) dst[i] = src[i];
  }
  __syncthreads();
  const int p[3] = {d.lo[0] + (int)(blockIdx.x * blockDim.x + threadIdx.x),
                    d.lo[1] + (int)(blockIdx.y * blockDim.y + threadIdx.y),
                    d.lo[2] + (int)(blockIdx.z * blockDim.z + threadIdx.z)};
  if (p[0] >= d.hi[0] || p[1] >= d.hi[1] || p[2] >= d.hi[2]) return;
  if (color >= 0 && ((p[0] + p[1] + p[2] + color) & 1)) return;
  A acc = 0;
  for (int i = 0; i < t.nterms; i++) {
    A v = xmul(gen_factor<A>(G, t.a[i], p), gen_factor<A>(G, t.b[i], p));
    acc = i ? xadd(acc, v) : v;
  }
  if (t.has_post) acc = xmul(acc, gen_factor<A>(G, t.post, p));
  GenFactor self;
  self.grid = G.out;
  self.off[0] = self.off[1] = self.off[2] = 0;
  self.boundary = PSB_BOUNDARY_NONE;
  const GridView &og = G.g[G.out];
  gen_store<A>(og, gen_offset(og, G.axes[G.out], G.nd[G.out], self, p), acc);
}

static GenFactor compact(const psb_factor &f) {
  GenFactor g;
  g.grid = f.grid;
  for (int i = 0; i < 3; i++) g.off[i] = f.offset[i];
  g.boundary = f.boundary;
  g.c = f.constant;
  return g;
}

psb_status generic_upload(GenericDesc &d) {
  GenTable t;
  memset(&t, 0, sizeof(t));
  t.nterms = d.host.nterms;
  t.has_post = d.host.has_post;
  t.post = compact(d.host.post);
  for (int i = 0; i < d.host.nterms; i++) {
    t.a[i] = compact(d.host.terms[i].a);
    t.b[i] = compact(d.host.terms[i].b);
  }
  if (!d.dev) PSB_TRY(cudaMalloc(&d.dev, sizeof(GenTable)));
  PSB_TRY(cudaMemcpy(d.dev, &t, sizeof(t), cudaMemcpyHostToDevice));
  return PSB_OK;
}

psb_status generic_launch(MapImpl &m, const GenericDesc &gd, int color, cudaStream_t s,
                          int64_t *launches) {
  // The TMA z-streaming kernel takes every map it can (k_generic_tma.cu);
  // PSB_IMPL_PLAIN and PSB_IMPL_GENERIC keep the thread-per-point kernel.
  if (rt().impl != PSB_IMPL_PLAIN && rt().impl != PSB_IMPL_GENERIC) {
    const psb_status st = generic_tma_launch(m, gd, color, s, launches);
    if (st != PSB_ERR_UNSUPPORTED) return st;
  }
  generic_note_impl(PSB_IMPL_GENERIC);
  const psb_generic_stencil &desc = gd.host;
  GenGrids G;
  for (int i = 0; i < desc.ngrids; i++) {
    G.g[i] = m.grids[i]->view();
    G.g[i].type = desc.grid_type[i];
    G.nd[i] = 0;
    for (int k = 0; k < 3; k++) {
      G.axes[i][k] = desc.grid_axes[i][k];
      if (desc.grid_axes[i][k] >= 0) G.nd[i] = k + 1;
    }
  }
  G.out = desc.out_grid;
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    d.lo[i] = i < desc.ndims ? m.dom.local_min[i] : 0;
    d.hi[i] = i < desc.ndims ? m.dom.local_max[i] : 1;
  }
  int ext[3] = {d.hi[0] - d.lo[0], d.hi[1] - d.lo[1], d.hi[2] - d.lo[2]};
  if (ext[0] <= 0 || ext[1] <= 0 || ext[2] <= 0) return PSB_OK;
  dim3 block(ext[0] >= 32 ? 32 : (ext[0] >= 16 ? 16 : 8), ext[1] >= 4 ? 4 : 1, 1);
  if (block.x * block.y < 64 && ext[2] > 1) block.z = 2;
  dim3 grid((ext[0] + block.x - 1) / block.x, (ext[1] + block.y - 1) / block.y,
            (ext[2] + block.z - 1) / block.z);
  if (grid.y > 65535 || grid.z > 65535) return set_status(PSB_ERR_INVALID);
  const GenTable *tab = (const GenTable *)gd.dev;
  switch (desc.accum_type) {
    case PS_FLOAT: k_generic<float><<<grid, block, 0, s>>>(tab, G, d, color); break;
    case PS_DOUBLE: k_generic<double><<<grid, block, 0, s>>>(tab, G, d, color); break;
    case PS_INT: k_generic<int32_t><<<grid, block, 0, s>>>(tab, G, d, color); break;
    default: k_generic<int64_t><<<grid, block, 0, s>>>(tab, G, d, color); break;
  }
  (*launches)++;
  return PSB_OK;
}

// --------------------------------------------------------------------------
// Kernel-function reduction: the value a generic stencil would emit at each
// point of the domain (evaluated exactly as k_generic does, converted to the
// emitted grid's element type) is reduced instead of stored -- the
// PSReduce(&v, op, kernel, dom, ...) form of the reference's documentation
// (docs/programming.md:298-320; the reference leaves it unimplemented,
// translator/reference_translator.cc:1357-1360). One pass, no temporary
// grid: each warp walks x rows of the domain, values accumulate in FP64
// (SUM compensated), CTAs combine in index order through the same scratch
// as the grid reduction.
// --------------------------------------------------------------------------
__device__ __forceinline__ double as_emitted(int type, double v) {
  switch (type) {
    case PS_FLOAT: return (double)(float)v;
    case PS_INT: return (double)(int32_t)v;
    case PS_LONG: return (double)(int64_t)v;
    default: return v;
  }
}

template <typename A>
__global__ void __launch_bounds__(256) k_generic_reduce(const GenTable *__restrict__ tab,
                                                        GenGrids G, Dom3 d, int op,
                                                        ReduceScratch sc) {
  __shared__ GenTable t;
  __shared__ RAcc scratch[32];
  __shared__ int is_last;
  {
    const int words = sizeof(GenTable) / 4;
    const uint32_t *src = reinterpret_cast<const uint32_t *>(tab);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&t);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int out_type = G.g[G.out].type;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int rx = d.hi[0] - d.lo[0], ry = d.hi[1] - d.lo[1];
  const int64_t rows = (int64_t)ry * (d.hi[2] - d.lo[2]);
  RAcc a = racc_init(op);
  for (int64_t r = warp; r < rows; r += nwarps) {
    int p[3];
    p[1] = d.lo[1] + (int)(r % ry);
    p[2] = d.lo[2] + (int)(r / ry);
    for (int x = lane; x < rx; x += 32) {
      p[0] = d.lo[0] + x;
      A acc = 0;
      for (int i = 0; i < t.nterms; i++) {
        A v = xmul(gen_factor<A>(G, t.a[i], p), gen_factor<A>(G, t.b[i], p));
        acc = i ? xadd(acc, v) : v;
      }
      if (t.has_post) acc = xmul(acc, gen_factor<A>(G, t.post, p));
      racc_add(op, a, as_emitted(out_type, (double)acc));
    }
  }
  RAcc b = racc_block(op, a, scratch);
  if (threadIdx.x == 0) {
    sc.partials[blockIdx.x] = b;
    __threadfence();
    const unsigned tk = atomicAdd(sc.ticket, 1u);
    is_last = (tk == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  RAcc acc = racc_init(op);
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
    RAcc q;
    q.s = __ldcg(&sc.partials[i].s);
    q.c = __ldcg(&sc.partials[i].c);
    acc = racc_merge(op, acc, q);
  }
  RAcc tot = racc_block(op, acc, scratch);
  if (threadIdx.x == 0) {
    *sc.result = op == PS_SUM ? tot.s + tot.c : tot.s;
    *sc.ticket = 0;
  }
}

psb_status generic_reduce(MapImpl &m, const GenericDesc &gd, int op, double *result,
                          cudaStream_t s) {
  const psb_generic_stencil &desc = gd.host;
  GenGrids G;
  for (int i = 0; i < desc.ngrids; i++) {
    G.g[i] = m.grids[i]->view();
    G.g[i].type = desc.grid_type[i];
    G.nd[i] = 0;
    for (int k = 0; k < 3; k++) {
      G.axes[i][k] = desc.grid_axes[i][k];
      if (desc.grid_axes[i][k] >= 0) G.nd[i] = k + 1;
    }
  }
  G.out = desc.out_grid;
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    d.lo[i] = i < desc.ndims ? m.dom.local_min[i] : 0;
    d.hi[i] = i < desc.ndims ? m.dom.local_max[i] : 1;
  }
  const int64_t rows = (int64_t)(d.hi[1] - d.lo[1]) * (d.hi[2] - d.lo[2]);
  if (rows <= 0 || d.hi[0] <= d.lo[0]) return set_status(PSB_ERR_INVALID);
  ReduceScratch sc;
  PSB_CHECK(reduce_scratch(&sc));
  const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((rows + 7) / 8, kReduceMaxBlocks));
  const GenTable *tab = (const GenTable *)gd.dev;
  switch (desc.accum_type) {
    case PS_FLOAT: k_generic_reduce<float><<<blocks, 256, 0, s>>>(tab, G, d, op, sc); break;
    case PS_DOUBLE: k_generic_reduce<double><<<blocks, 256, 0, s>>>(tab, G, d, op, sc); break;
    case PS_INT: k_generic_reduce<int32_t><<<blocks, 256, 0, s>>>(tab, G, d, op, sc); break;
    default: k_generic_reduce<int64_t><<<blocks, 256, 0, s>>>(tab, G, d, op, sc); break;
  }
  PSB_TRY(cudaGetLastError());
  PSB_TRY(cudaMemcpyAsync(result, sc.result, sizeof(double), cudaMemcpyDeviceToHost, s));
  PSB_TRY(cudaStreamSynchronize(s));
  return PSB_OK;
}

// --------------------------------------------------------------------------
// Halo fill: ghost cells of a pitched grid from the periodic (mode 1) or
// clamped (mode 2) image of the interior. The ghost shell is enumerated as
// z slabs (full x-y extent), then y slabs (interior z), then x slabs.
// --------------------------------------------------------------------------
template <typename T>
__global__ void k_halo_fill(GridView g, int hx, int hy, int hz, int mode) {
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t ex = nx + 2 * hx, ey = ny + 2 * hy;
  const int64_t A = (int64_t)2 * hz * ey * ex;
  const int64_t B = (int64_t)nz * 2 * hy * ex;
  const int64_t C = (int64_t)nz * ny * 2 * hx;
  const int64_t total = A + B + C;
  T *o = (T *)g.origin;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    if (i < A) {
      int64_t r = i;
      x = (int)(r % ex) - hx;
      r /= ex;
      y = (int)(r % ey) - hy;
      r /= ey;
      int zz = (int)r;  // 0 .. 2hz-1
      z = zz < hz ? zz - hz : nz + (zz - hz);
    } else if (i < A + B) {
      int64_t r = i - A;
      x = (int)(r % ex) - hx;
      r /= ex;
      int yy = (int)(r % (2 * hy));
      y = yy < hy ? yy - hy : ny + (yy - hy);
      z = (int)(r / (2 * hy));
    } else {
      int64_t r = i - A - B;
      int xx = (int)(r % (2 * hx));
      x = xx < hx ? xx - hx : nx + (xx - hx);
      r /= 2 * hx;
      y = (int)(r % ny);
      z = (int)(r / ny);
    }
    int sx, sy_, sz_;
    if (mode == PSB_BOUNDARY_PERIODIC) {
      sx = ((x % nx) + nx) % nx;
      sy_ = ((y % ny) + ny) % ny;
      sz_ = ((z % nz) + nz) % nz;
    } else {
      sx = min(max(x, 0), nx - 1);
      sy_ = min(max(y, 0), ny - 1);
      sz_ = min(max(z, 0), nz - 1);
    }
    o[(int64_t)x + y * g.sy + z * g.sz] = o[(int64_t)sx + sy_ * g.sy + sz_ * g.sz];
  }
}

psb_status launch_halo_fill(GridImpl *gi, int mode, cudaStream_t s) {
  if (gi->layout != PSB_LAYOUT_PITCHED) return PSB_OK;
  GridView v = gi->view();
  int nd = gi->pub.num_dims;
  int hx = gi->halo, hy = nd > 1 ? gi->halo : 0, hz = nd > 2 ? gi->halo : 0;
  int threads = 256;
  int64_t total = (int64_t)2 * hz * (v.n[1] + 2 * hy) * (v.n[0] + 2 * hx) +
                  (int64_t)v.n[2] * 2 * hy * (v.n[0] + 2 * hx) + (int64_t)v.n[2] * v.n[1] * 2 * hx;
  int blocks = (int)std::min<int64_t>((total + threads - 1) / threads, rt().sm_count * 16);
  if (blocks < 1) blocks = 1;
  if (gi->pub.elm_size == 8)
    k_halo_fill<double><<<blocks, threads, 0, s>>>(v, hx, hy, hz, mode);
  else
    k_halo_fill<float><<<blocks, threads, 0, s>>>(v, hx, hy, hz, mode);
  gi->ghost_valid = mode;
  return PSB_OK;
}

}  // namespace psb
