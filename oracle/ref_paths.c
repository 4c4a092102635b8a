/*
 * oracle/ref_paths.c -- the reference CPU target running the benchmark
 * stencils, for parity checks and the CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY (never linked into the product). Compiled against
 * the reference's own headers (include/physis/physis_ref.h) and linked with
 * libphysis_rt_ref built from the reference's runtime sources by
 * oracle/Makefile. The functions below are written in the shape that the
 * reference translator emits for the ref target, because the translator
 * itself (ROSE) cannot be built here:
 *  - the stencil function becomes an inline C function whose gets are
 *    ((T*)g->p0)[__PSGridGetOffset3D(g, ...)] and whose emit writes g->p0
 *    (translator/reference_runtime_builder.cc:72-176,
 *     reference_translator.cc:161-165);
 *  - a run-kernel function loops k/j/i, i innermost, over
 *    [local_min, local_max-1] (reference_translator.cc:479-549);
 *  - __PSStencilRun_N(iter, s0, s1) calls the run kernels in order iter
 *    times (reference_translator.cc:697-747).
 * Grid allocation, copy-in/out and PSReduce are the reference runtime's own
 * code (runtime/libphysis_rt_ref.cc). Stencil bodies restate the DSL
 * sources examples/diffusion-benchmark/diffusion3d_physis.c:29-58 and
 * examples/himeno/himenobmtxpa_physis.c:331-361 in that lowered form.
 */
#define PHYSIS_REF 1
#include <time.h>
#include "physis/physis_ref.h"

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}

/* ---------------- 7-point diffusion, clamped and periodic ---------------- */
#define DEFINE_DIFF(SUFFIX, REAL)                                               \
  typedef struct {                                                             \
    __PSDomain dom;                                                            \
    __PSGrid *g1;                                                              \
    int g1_index;                                                              \
    __PSGrid *g2;                                                              \
    int g2_index;                                                              \
    REAL ce, cw, cn, cs, ct, cb, cc;                                           \
  } __PSStencil_diff_##SUFFIX;                                                 \
  static inline void diff_kernel_##SUFFIX(const int x, const int y,           \
                                          const int z, __PSGrid *g1,           \
                                          __PSGrid *g2, REAL ce, REAL cw,      \
                                          REAL cn, REAL cs, REAL ct, REAL cb,  \
                                          REAL cc) {                           \
    int nx = PSGridDim(g1, 0), ny = PSGridDim(g1, 1), nz = PSGridDim(g1, 2);   \
    REAL c, w, e, n, s, b, t;                                                  \
    c = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y, z)];                    \
    if (x == 0) w = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y, z)];        \
    else w = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x - 1, y, z)];           \
    if (x == nx - 1) e = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y, z)];   \
    else e = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x + 1, y, z)];           \
    if (y == 0) n = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y, z)];        \
    else n = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y - 1, z)];           \
    if (y == ny - 1) s = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y, z)];   \
    else s = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y + 1, z)];           \
    if (z == 0) b = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y, z)];        \
    else b = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y, z - 1)];           \
    if (z == nz - 1) t = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y, z)];   \
    else t = ((REAL *)g1->p0)[__PSGridGetOffset3D(g1, x, y, z + 1)];           \
    ((REAL *)g2->p0)[__PSGridGetOffset3D(g2, x, y, z)] =                       \
        cc * c + cw * w + ce * e + cs * s + cn * n + cb * b + ct * t;          \
  }                                                                            \
  static inline void diffp_kernel_##SUFFIX(const int x, const int y,          \
                                           const int z, __PSGrid *g1,          \
                                           __PSGrid *g2, REAL ce, REAL cw,     \
                                           REAL cn, REAL cs, REAL ct, REAL cb, \
                                           REAL cc) {                          \
    REAL c = ((REAL *)g1->p0)[__PSGridGetOffsetPeriodic3D(g1, x, y, z)];       \
    REAL w = ((REAL *)g1->p0)[__PSGridGetOffsetPeriodic3D(g1, x - 1, y, z)];   \
    REAL e = ((REAL *)g1->p0)[__PSGridGetOffsetPeriodic3D(g1, x + 1, y, z)];   \
    REAL n = ((REAL *)g1->p0)[__PSGridGetOffsetPeriodic3D(g1, x, y - 1, z)];   \
    REAL s = ((REAL *)g1->p0)[__PSGridGetOffsetPeriodic3D(g1, x, y + 1, z)];   \
    REAL b = ((REAL *)g1->p0)[__PSGridGetOffsetPeriodic3D(g1, x, y, z - 1)];   \
    REAL t = ((REAL *)g1->p0)[__PSGridGetOffsetPeriodic3D(g1, x, y, z + 1)];   \
    ((REAL *)g2->p0)[__PSGridGetOffset3D(g2, x, y, z)] =                       \
        cc * c + cw * w + ce * e + cs * s + cn * n + cb * b + ct * t;          \
  }                                                                            \
  static void __PSStencilRun_kernel_diff_##SUFFIX(                             \
      const __PSStencil_diff_##SUFFIX *s, int periodic) {                      \
    int i0, i1, i2;                                                            \
    for (i2 = s->dom.local_min[2]; i2 <= s->dom.local_max[2] - 1; i2++)        \
      for (i1 = s->dom.local_min[1]; i1 <= s->dom.local_max[1] - 1; i1++)      \
        for (i0 = s->dom.local_min[0]; i0 <= s->dom.local_max[0] - 1; i0++) {  \
          if (periodic)                                                        \
            diffp_kernel_##SUFFIX(i0, i1, i2, s->g1, s->g2, s->ce, s->cw,     \
                                  s->cn, s->cs, s->ct, s->cb, s->cc);          \
          else                                                                 \
            diff_kernel_##SUFFIX(i0, i1, i2, s->g1, s->g2, s->ce, s->cw,      \
                                 s->cn, s->cs, s->ct, s->cb, s->cc);           \
        }                                                                      \
  }                                                                            \
  static float __PSStencilRun_diff_##SUFFIX(int iter,                         \
                                            __PSStencil_diff_##SUFFIX s0,      \
                                            __PSStencil_diff_##SUFFIX s1,      \
                                            int periodic) {                    \
    int i;                                                                     \
    for (i = 0; i < iter; ++i) {                                               \
      __PSStencilRun_kernel_diff_##SUFFIX(&s0, periodic);                      \
      __PSStencilRun_kernel_diff_##SUFFIX(&s1, periodic);                      \
    }                                                                          \
    return 0.0f;                                                               \
  }                                                                            \
  /* count double-buffered steps (count even) on an nx*ny*nz field: copy-in,  \
     run(count/2) of (g1->g2, g2->g1), copy-out of g1. Returns the seconds    \
     spent in the run loop only (copy-in/out excluded). */                     \
  double refp_diffusion7_##SUFFIX(int nx, int ny, int nz, REAL *field,         \
                                  int count, const REAL *coef, int periodic) { \
    PSVectorInt dims = {nx, ny, nz};                                           \
    __PSGrid *g1 = __PSGridNew(sizeof(REAL), 3, dims);                         \
    __PSGrid *g2 = __PSGridNew(sizeof(REAL), 3, dims);                         \
    PSDomain3D dom = PSDomain3DNew(0, nx, 0, ny, 0, nz);                       \
    PSGridCopyin(g1, field);                                                   \
    __PSStencil_diff_##SUFFIX s0 = {dom, g1, 0, g2, 0, coef[0], coef[1],       \
                                    coef[2], coef[3], coef[4], coef[5],        \
                                    coef[6]};                                  \
    __PSStencil_diff_##SUFFIX s1 = s0;                                         \
    s1.g1 = g2;                                                                \
    s1.g2 = g1;                                                                \
    double t0 = now_s();                                                       \
    __PSStencilRun_diff_##SUFFIX(count / 2, s0, s1, periodic);                 \
    double t1 = now_s();                                                       \
    PSGridCopyout(g1, field);                                                  \
    PSGridFree(g1);                                                            \
    PSGridFree(g2);                                                            \
    free(g1);                                                                  \
    free(g2);                                                                  \
    return t1 - t0;                                                            \
  }

DEFINE_DIFF(f32, float)
DEFINE_DIFF(f64, double)

/* ---------------- Himeno 19-point Jacobi ---------------- */
typedef struct {
  __PSDomain dom;
  __PSGrid *p0, *p1, *a0, *a1, *a2, *a3, *b0, *b1, *b2, *c0, *c1, *c2, *bnd, *wrk1;
  float omega;
} __PSStencil_jacobi;

#define G(g, i, j, k) (((float *)(g)->p0)[__PSGridGetOffset3D((g), (i), (j), (k))])

static inline void jacobi_kernel(int i, int j, int k, const __PSStencil_jacobi *s) {
  float s0, ss;
  s0 = G(s->a0, i, j, k) * G(s->p0, i, j, k + 1) +
       G(s->a1, i, j, k) * G(s->p0, i, j + 1, k) +
       G(s->a2, i, j, k) * G(s->p0, i + 1, j, k) +
       G(s->b0, i, j, k) * (G(s->p0, i, j + 1, k + 1) - G(s->p0, i, j - 1, k + 1) -
                            G(s->p0, i, j + 1, k - 1) + G(s->p0, i, j - 1, k - 1)) +
       G(s->b1, i, j, k) * (G(s->p0, i + 1, j + 1, k) - G(s->p0, i + 1, j - 1, k) -
                            G(s->p0, i - 1, j + 1, k) + G(s->p0, i - 1, j - 1, k)) +
       G(s->b2, i, j, k) * (G(s->p0, i + 1, j, k + 1) - G(s->p0, i + 1, j, k - 1) -
                            G(s->p0, i - 1, j, k + 1) + G(s->p0, i - 1, j, k - 1)) +
       G(s->c0, i, j, k) * G(s->p0, i, j, k - 1) +
       G(s->c1, i, j, k) * G(s->p0, i, j - 1, k) +
       G(s->c2, i, j, k) * G(s->p0, i - 1, j, k) + G(s->wrk1, i, j, k);
  ss = (s0 * G(s->a3, i, j, k) - G(s->p0, i, j, k)) * G(s->bnd, i, j, k);
  float v = G(s->p0, i, j, k) + s->omega * ss;
  G(s->p1, i, j, k) = v;
}

static void __PSStencilRun_kernel_jacobi(const __PSStencil_jacobi *s) {
  int i0, i1, i2;
  for (i2 = s->dom.local_min[2]; i2 <= s->dom.local_max[2] - 1; i2++)
    for (i1 = s->dom.local_min[1]; i1 <= s->dom.local_max[1] - 1; i1++)
      for (i0 = s->dom.local_min[0]; i0 <= s->dom.local_max[0] - 1; i0++)
        jacobi_kernel(i0, i1, i2, s);
}

static float __PSStencilRun_jacobi(int iter, __PSStencil_jacobi s0, __PSStencil_jacobi s1) {
  int i;
  for (i = 0; i < iter; ++i) {
    __PSStencilRun_kernel_jacobi(&s0);
    __PSStencilRun_kernel_jacobi(&s1);
  }
  return 0.0f;
}

/* nn sweeps (even) of the Himeno update on an nx*ny*nz problem. p holds the
 * initial pressure on entry and the result on exit; coef[0..11] are the
 * host fields a0 a1 a2 a3 b0 b1 b2 c0 c1 c2 bnd wrk1. p1 starts as a copy of
 * p, as in himenobmtxpa_physis.c:137-138. Returns run-loop seconds. */
double refp_himeno_f32(int nx, int ny, int nz, float *p, const float *const *coef,
                       float omega, int nn) {
  PSVectorInt dims = {nx, ny, nz};
  __PSGrid *g[14];
  for (int i = 0; i < 14; i++) g[i] = __PSGridNew(sizeof(float), 3, dims);
  PSGridCopyin(g[0], p);
  PSGridCopyin(g[1], p);
  for (int i = 0; i < 12; i++) PSGridCopyin(g[2 + i], coef[i]);
  PSDomain3D inner = PSDomain3DNew(1, nx - 1, 1, ny - 1, 1, nz - 1);
  __PSStencil_jacobi s0 = {inner, g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7],
                           g[8], g[9], g[10], g[11], g[12], g[13], omega};
  __PSStencil_jacobi s1 = s0;
  s1.p0 = g[1];
  s1.p1 = g[0];
  double t0 = now_s();
  __PSStencilRun_jacobi(nn / 2, s0, s1);
  double t1 = now_s();
  PSGridCopyout(g[0], p);
  for (int i = 0; i < 14; i++) {
    PSGridFree(g[i]);
    free(g[i]);
  }
  return t1 - t0;
}

/* ---------------- 27-point box average (a user stencil) ---------------- */
/* The stencil of tests/system_tests/test_cases/test_27-pt.c (neighbours in
 * its order: z = -1, 0, 1, and in each plane the centre, then x+1, x-1,
 * y+1 with its corners, y-1 with its corners), each neighbour weighted by
 * c, in the ref target's lowered form; domain [1, n-1) per axis. */
typedef struct {
  __PSDomain dom;
  __PSGrid *g1;
  int g1_index;
  __PSGrid *g2;
  int g2_index;
  float c;
} __PSStencil_box27;

#define B27(g, i, j, k) (((float *)(g)->p0)[__PSGridGetOffset3D((g), (i), (j), (k))])
#define B27_PLANE(g, i, j, k, c)                                                          \
  c * B27(g, i, j, k) + c * B27(g, i + 1, j, k) + c * B27(g, i - 1, j, k) +               \
      c * B27(g, i, j + 1, k) + c * B27(g, i + 1, j + 1, k) + c * B27(g, i - 1, j + 1, k) + \
      c * B27(g, i, j - 1, k) + c * B27(g, i + 1, j - 1, k) + c * B27(g, i - 1, j - 1, k)

static inline void box27_kernel(int i, int j, int k, __PSGrid *g1, __PSGrid *g2, float c) {
  B27(g2, i, j, k) = B27_PLANE(g1, i, j, k - 1, c) + B27_PLANE(g1, i, j, k, c) +
                     B27_PLANE(g1, i, j, k + 1, c);
}

static void __PSStencilRun_kernel_box27(const __PSStencil_box27 *s) {
  int i0, i1, i2;
  for (i2 = s->dom.local_min[2]; i2 <= s->dom.local_max[2] - 1; i2++)
    for (i1 = s->dom.local_min[1]; i1 <= s->dom.local_max[1] - 1; i1++)
      for (i0 = s->dom.local_min[0]; i0 <= s->dom.local_max[0] - 1; i0++)
        box27_kernel(i0, i1, i2, s->g1, s->g2, s->c);
}

/* count (even) double-buffered steps; both grids start as `field` (the
 * boundary cells keep it). Returns run-loop seconds. */
double refp_box27_f32(int nx, int ny, int nz, float *field, int count, float c) {
  PSVectorInt dims = {nx, ny, nz};
  __PSGrid *g1 = __PSGridNew(sizeof(float), 3, dims);
  __PSGrid *g2 = __PSGridNew(sizeof(float), 3, dims);
  PSGridCopyin(g1, field);
  PSGridCopyin(g2, field);
  PSDomain3D inner = PSDomain3DNew(1, nx - 1, 1, ny - 1, 1, nz - 1);
  __PSStencil_box27 s0 = {inner, g1, 0, g2, 0, c};
  __PSStencil_box27 s1 = s0;
  s1.g1 = g2;
  s1.g2 = g1;
  double t0 = now_s();
  for (int it = 0; it < count / 2; ++it) {
    __PSStencilRun_kernel_box27(&s0);
    __PSStencilRun_kernel_box27(&s1);
  }
  double t1 = now_s();
  PSGridCopyout(g1, field);
  PSGridFree(g1);
  PSGridFree(g2);
  free(g1);
  free(g2);
  return t1 - t0;
}

/* ---------------- PSReduce through the reference runtime ---------------- */
void refp_reduce_f32(int op, const float *data, int64_t n, float *out) {
  PSVectorInt dims = {(int)n, 1, 1};
  __PSGrid *g = __PSGridNew(sizeof(float), 1, dims);
  PSGridCopyin(g, data);
  __PSReduceGridFloat(out, (enum PSReduceOp)op, g);
  PSGridFree(g);
  free(g);
}
void refp_reduce_f64(int op, const double *data, int64_t n, double *out) {
  PSVectorInt dims = {(int)n, 1, 1};
  __PSGrid *g = __PSGridNew(sizeof(double), 1, dims);
  PSGridCopyin(g, data);
  __PSReduceGridDouble(out, (enum PSReduceOp)op, g);
  PSGridFree(g);
  free(g);
}

/* PSInit of the ref target, once per process (runtime/libphysis_rt_ref.cc:45-50). */
void refp_init(void) {
  static int done = 0;
  if (done) return;
  int argc = 1;
  char *args[] = {(char *)"oracle", NULL};
  char **argv = args;
  PSInit(&argc, &argv, 3, 1, 1, 1);
  done = 1;
}
