// Seeded synthetic fields generated on the device (benchmarks and tests fill
// tens of GB of grids; generating them on the host would dominate the run).
//
// Element (x, y, z) of a fill with seed s takes the 64-bit hash
// h = splitmix64(s * 0x9E3779B97F4A7C15 + (x + nx*(y + ny*z)))  and
//   kind 0: lo + (hi - lo) * u,  u = (h >> 40) * 2^-24  (uniform [lo, hi))
//   kind 1: lo                                         (constant)
//   kind 2: 1 inside, 0 on the faces                   (Himeno bnd)
//   kind 3: (z / (nz - 1))^2                           (Himeno initial p)
// computed in double and rounded to the grid's type once.
#include "device.cuh"

namespace psb {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

template <typename T>
__global__ void k_fill(GridView g, int kind, uint64_t seed, double lo, double hi) {
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t total = (int64_t)nx * ny * nz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const int64_t r = i / nx;
    const int y = (int)(r % ny);
    const int z = (int)(r / ny);
    double v;
    switch (kind) {
      case 0: {
        const uint64_t h = splitmix64(seed * 0x9E3779B97F4A7C15ull + (uint64_t)i);
        v = lo + (hi - lo) * ((double)(h >> 40) * (1.0 / 16777216.0));
        break;
      }
      case 1: v = lo; break;
      case 2:
        v = (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1) ? 0.0 : 1.0;
        break;
      default: {
        const double t = nz > 1 ? (double)z / (double)(nz - 1) : 0.0;
        v = t * t;
        break;
      }
    }
    ((T *)g.origin)[(int64_t)x + (int64_t)y * g.sy + (int64_t)z * g.sz] = (T)v;
  }
}

}  // namespace psb

using namespace psb;

extern "C" psb_status psb_grid_fill(__PSGrid *p, int kind, uint64_t seed, double lo, double hi) {
  GridImpl *g = as_impl(p);
  if (!g || g->user_type || kind < 0 || kind > 3) return set_status(PSB_ERR_INVALID);
  PSB_CHECK(ensure_init());
  Runtime &r = rt();
  GridView v = g->view();
  const int64_t total = (int64_t)v.n[0] * v.n[1] * v.n[2];
  const int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)r.sm_count * 16);
  switch (g->type) {
    case PS_FLOAT: k_fill<float><<<blocks, 256, 0, r.stream>>>(v, kind, seed, lo, hi); break;
    case PS_DOUBLE: k_fill<double><<<blocks, 256, 0, r.stream>>>(v, kind, seed, lo, hi); break;
    case PS_INT: k_fill<int32_t><<<blocks, 256, 0, r.stream>>>(v, kind, seed, lo, hi); break;
    case PS_LONG: k_fill<int64_t><<<blocks, 256, 0, r.stream>>>(v, kind, seed, lo, hi); break;
    default: return set_status(PSB_ERR_INVALID);
  }
  PSB_TRY(cudaGetLastError());
  if (g->layout == PSB_LAYOUT_PITCHED) g->ghost_valid = PSB_BOUNDARY_NONE;
  return PSB_OK;
}
