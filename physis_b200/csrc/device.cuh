// Device helpers shared by the kernels: exact arithmetic, TMA/mbarrier PTX,
// bounded waits and periodic halo images.
#pragma once

#ifdef __CUDACC_RTC__
// Compiled at run time: the library hands the compiler the fixed-width
// integer types and the tensor-map type itself (rtc.cu).
#include "psb_rtc_prelude.h"
#include "views.h"
#else
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"
#endif

namespace psb {

// Round-to-nearest multiply and add that the compiler never contracts into
// an FMA: with these, a kernel computes a*b + c*d ... with exactly the
// roundings of the reference CPU target built with -ffp-contract=off.
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ int32_t xmul(int32_t a, int32_t b) { return a * b; }
__device__ __forceinline__ int64_t xmul(int64_t a, int64_t b) { return a * b; }
__device__ __forceinline__ int32_t xadd(int32_t a, int32_t b) { return a + b; }
__device__ __forceinline__ int64_t xadd(int64_t a, int64_t b) { return a + b; }

// Vector of 16 bytes of T (4 floats or 2 doubles).
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  static constexpr int N = 4;
  float v[4];
};
template <>
struct Vec16<double> {
  static constexpr int N = 2;
  double v[2];
};

template <typename T>
__device__ __forceinline__ Vec16<T> lds16(const T *p) {
  Vec16<T> r;
  if constexpr (sizeof(T) == 4) {
    float4 q = *reinterpret_cast<const float4 *>(p);
    r.v[0] = q.x; r.v[1] = q.y; r.v[2] = q.z; r.v[3] = q.w;
  } else {
    double2 q = *reinterpret_cast<const double2 *>(p);
    r.v[0] = q.x; r.v[1] = q.y;
  }
  return r;
}

template <typename T>
__device__ __forceinline__ void stg16(T *p, const Vec16<T> &r) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
  } else {
    *reinterpret_cast<double2 *>(p) = make_double2(r.v[0], r.v[1]);
  }
}

// Streaming 16-byte global load that does not allocate in L1 (coefficient
// fields are read exactly once per sweep).
template <typename T>
__device__ __forceinline__ Vec16<T> ldg16_stream(const T *p) {
  Vec16<T> r;
  if constexpr (sizeof(T) == 4) {
    float4 q = __ldcs(reinterpret_cast<const float4 *>(p));
    r.v[0] = q.x; r.v[1] = q.y; r.v[2] = q.z; r.v[3] = q.w;
  } else {
    double2 q = __ldcs(reinterpret_cast<const double2 *>(p));
    r.v[0] = q.x; r.v[1] = q.y;
  }
  return r;
}

// ---------------------------------------------------------------------------
// mbarrier + TMA (sm_90+ PTX, used here on sm_100a). No cluster multicast.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// try_wait with a suspend-time hint (ns): a waiting warp sleeps in the
// barrier unit instead of spinning through issue slots.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(1000000u)
      : "memory");
  return ok != 0;
}

// Wait for the barrier phase with a clock bound (~1.5 s at 1.9 GHz). Returns
// false if it gave up; the caller then records an error and leaves.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait_sleep(bar, parity)) return true;
  long long t0 = clock64();
  while (!mbar_try_wait_sleep(bar, parity)) {
    if (clock64() - t0 > 3000000000LL) return false;
  }
  return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 3-D tiled TMA load of one box into shared memory, completing on bar.
// Coordinates are in elements; x * sizeof(T) must be a multiple of 16.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Bring one box of a tensor into L2 (no shared memory, no completion).
__device__ __forceinline__ void tma_prefetch_l2_3d(const CUtensorMap *map, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z)
               : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Face images for the 7-point stencil: it only reads the six face
// neighbours, so the halo cells it needs are the depth-1 faces (x = -1 and
// x = n at interior y, z, and likewise for y and z). A writer of interior
// point (x, y, z) keeps them periodic by storing its value at the face image
// of each axis where it lies on the opposite face.
template <typename T>
__device__ __forceinline__ void store_face_images(T *origin, int64_t sy, int64_t sz, const int *n,
                                                  int x, int y, int z, T v) {
  const int64_t c = (int64_t)x + y * sy + z * sz;
  if (x == 0) origin[c + n[0]] = v;
  if (x == n[0] - 1) origin[c - n[0]] = v;
  if (y == 0) origin[c + n[1] * sy] = v;
  if (y == n[1] - 1) origin[c - n[1] * sy] = v;
  if (z == 0) origin[c + n[2] * sz] = v;
  if (z == n[2] - 1) origin[c - n[2] * sz] = v;
}

// A ring of S shared-memory stages filled by TMA (one producer thread) and
// drained by consumer warps. The position (slot, wrap count) is an explicit
// value, so one ring can carry the planes of many tiles back to back.
struct Ring {
  uint64_t *full;       // S barriers, one producer arrival (+ the copy's bytes)
  uint64_t *empty;      // S barriers, one arrival per consumer warp
  unsigned char *base;  // stage 0
  int S;
  int stage_bytes;
};

struct RingPos {
  int slot;
  uint32_t round;  // times the ring wrapped before this position
};

__device__ __forceinline__ void ring_next(RingPos &p, int S) {
  if (++p.slot == S) {
    p.slot = 0;
    p.round++;
  }
}

__device__ __forceinline__ void ring_init(const Ring &R, int consumer_warps) {
  for (int i = 0; i < R.S; i++) {
    mbar_init(&R.full[i], 1);
    mbar_init(&R.empty[i], consumer_warps);
  }
  mbar_fence_init();
}

// Producer: np planes, plane j from tensor coordinates (cx, cy, cz0 + j),
// into the ring from position p on. False if a bounded wait gave up.
__device__ __forceinline__ bool ring_produce(const Ring &R, RingPos &p, const CUtensorMap *tin,
                                             uint32_t bytes, int cx, int cy, int cz0, int np) {
  for (int j = 0; j < np; j++) {
    if (p.round > 0 && !mbar_wait_bounded(&R.empty[p.slot], (p.round - 1) & 1)) return false;
    mbar_arrive_expect_tx(&R.full[p.slot], bytes);
    tma_load_3d(R.base + p.slot * R.stage_bytes, tin, &R.full[p.slot], cx, cy, cz0 + j);
    ring_next(p, R.S);
  }
  return true;
}

// After a producer gave up: wait (bounded) until the last copy issued into
// each slot before position `end` has landed, so none is in flight when the
// CTA leaves.
__device__ __forceinline__ void ring_drain(const Ring &R, RingPos end) {
  for (int i = 0; i < R.S; i++) {
    if (end.round == 0 && i >= end.slot) continue;
    const uint32_t r = i < end.slot ? end.round : end.round - 1;
    const long long t0 = clock64();
    while (!mbar_try_wait(&R.full[i], r & 1) && clock64() - t0 < 200000000LL) {
    }
  }
}

}  // namespace psb
