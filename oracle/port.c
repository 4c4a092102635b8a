/*
 * oracle/port.c -- CPU restatement of the Physis stencil path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that the GPU runtime is
 * compared against; nothing in the product links, loads or calls it. Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * It restates, in plain C with the reference's loop order and arithmetic
 * order, what the reference CPU target computes:
 *  - loop nest k/j/i with i innermost over [local_min, local_max)
 *    (translator/reference_translator.cc:479-549);
 *  - get/emit lowered to dense x-fastest offsets x + y*nx + z*nx*ny and the
 *    periodic form ((i+n)%n) per axis (include/physis/physis_ref.h:57-79,
 *    translator/reference_runtime_builder.cc:72-176);
 *  - PSStencilRun(m0, m1, ..., iter): maps in order, iter times
 *    (reference_translator.cc:697-747);
 *  - PSReduce: a sequential left fold from d[0] (runtime/libphysis_rt_ref.cc:26-37)
 *    with the operators of runtime/reduce.h:19-55.
 * Build with -O2 -ffp-contract=off so no multiply-add is contracted; with
 * that, results are bit-identical to the reference CPU target.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/physis_b200.h"

#define IDX3(x, y, z, nx, ny) ((int64_t)(x) + (int64_t)(y) * (nx) + (int64_t)(z) * (int64_t)(nx) * (ny))

/* ------------------------------------------------------------------------ */
/* 7-point diffusion (examples/diffusion-benchmark/diffusion3d_physis.c:29-58) */
/* coef = {ce, cw, cn, cs, ct, cb, cc}: the kernel's parameter order.        */
/* out = cc*c + cw*w + ce*e + cs*s + cn*n + cb*b + ct*t (left to right).      */
/* periodic != 0 replaces the clamped neighbours by wrapped ones.            */
/* ------------------------------------------------------------------------ */
#define DEFINE_DIFFUSION7(NAME, REAL)                                          \
  static void NAME##_step(int nx, int ny, int nz, const REAL *g1, REAL *g2,    \
                          const REAL *cf, int periodic, const int *lo,          \
                          const int *hi) {                                      \
    const REAL ce = cf[0], cw = cf[1], cn = cf[2], cs = cf[3], ct = cf[4],      \
               cb = cf[5], cc = cf[6];                                          \
    for (int z = lo[2]; z < hi[2]; z++)                                         \
      for (int y = lo[1]; y < hi[1]; y++)                                       \
        for (int x = lo[0]; x < hi[0]; x++) {                                   \
          REAL c = g1[IDX3(x, y, z, nx, ny)];                                   \
          REAL w, e, n, s, b, t;                                                \
          if (periodic) {                                                       \
            w = g1[IDX3((x - 1 + nx) % nx, y, z, nx, ny)];                      \
            e = g1[IDX3((x + 1 + nx) % nx, y, z, nx, ny)];                      \
            n = g1[IDX3(x, (y - 1 + ny) % ny, z, nx, ny)];                      \
            s = g1[IDX3(x, (y + 1 + ny) % ny, z, nx, ny)];                      \
            b = g1[IDX3(x, y, (z - 1 + nz) % nz, nx, ny)];                      \
            t = g1[IDX3(x, y, (z + 1 + nz) % nz, nx, ny)];                      \
          } else {                                                              \
            w = (x == 0) ? c : g1[IDX3(x - 1, y, z, nx, ny)];                   \
            e = (x == nx - 1) ? c : g1[IDX3(x + 1, y, z, nx, ny)];              \
            n = (y == 0) ? c : g1[IDX3(x, y - 1, z, nx, ny)];                   \
            s = (y == ny - 1) ? c : g1[IDX3(x, y + 1, z, nx, ny)];              \
            b = (z == 0) ? c : g1[IDX3(x, y, z - 1, nx, ny)];                   \
            t = (z == nz - 1) ? c : g1[IDX3(x, y, z + 1, nx, ny)];              \
          }                                                                     \
          g2[IDX3(x, y, z, nx, ny)] =                                           \
              cc * c + cw * w + ce * e + cs * s + cn * n + cb * b + ct * t;     \
        }                                                                       \
  }                                                                             \
  /* steps single updates, ping-pong a -> b -> a ...; the result is left in a  \
     (copied back if steps is odd). Domain [lo, hi). */                         \
  void NAME(int nx, int ny, int nz, REAL *a, REAL *b, int steps,               \
            const REAL *coef, int periodic, const int *lo, const int *hi) {    \
    int full_lo[3] = {0, 0, 0}, full_hi[3] = {nx, ny, nz};                      \
    if (!lo) lo = full_lo;                                                      \
    if (!hi) hi = full_hi;                                                      \
    REAL *src = a, *dst = b;                                                    \
    for (int i = 0; i < steps; i++) {                                           \
      NAME##_step(nx, ny, nz, src, dst, coef, periodic, lo, hi);                \
      REAL *t = src;                                                            \
      src = dst;                                                                \
      dst = t;                                                                  \
    }                                                                           \
    if (src != a) memcpy(a, src, sizeof(REAL) * (size_t)nx * ny * nz);          \
  }

DEFINE_DIFFUSION7(orc_diffusion7_f32, float)
DEFINE_DIFFUSION7(orc_diffusion7_f64, double)

/* ------------------------------------------------------------------------ */
/* Himeno 19-point Jacobi (examples/himeno/himenobmtxpa_physis.c:331-361).   */
/* coef[0..13] = a0 a1 a2 a3 b0 b1 b2 c0 c1 c2 bnd wrk1 (12 used) -- order    */
/* of the kernel's grid parameters after p0, p1. One sweep over the interior */
/* [1, n-1) per axis writes p1 from p0. gosa (optional) receives, per sweep, */
/* sum of (double)ss*(double)ss over the interior, accumulated in FP64 in    */
/* loop order -- the residual of the original Himeno (gosa += ss*ss) carried */
/* in FP64.                                                                   */
/* ------------------------------------------------------------------------ */
/* The same sweep in REAL arithmetic: orc_himeno_f32 is the restatement of
 * the fp32 kernel; orc_himeno_f64 runs the identical expression tree in
 * double from inputs widened to double, the FP64 oracle against which the
 * error of an fp32 run is measured. */
#define DEFINE_HIMENO(NAME, REAL)                                              \
  void NAME(int nx, int ny, int nz, REAL *p0, REAL *p1,                        \
            const REAL *const *coef, REAL omega, int sweeps, double *gosa) {   \
    const REAL *a0 = coef[0], *a1 = coef[1], *a2 = coef[2], *a3 = coef[3];     \
    const REAL *b0 = coef[4], *b1 = coef[5], *b2 = coef[6];                    \
    const REAL *c0 = coef[7], *c1 = coef[8], *c2 = coef[9];                    \
    const REAL *bnd = coef[10], *wrk1 = coef[11];                              \
    REAL *src = p0, *dst = p1;                                                 \
    for (int it = 0; it < sweeps; it++) {                                      \
      /* gosa with Neumaier compensation so the checker is accurate to a few  \
         ulp whatever the summation order of the implementation under test */ \
      double g = 0.0, gc = 0.0;                                                \
      for (int k = 1; k < nz - 1; k++)                                         \
        for (int j = 1; j < ny - 1; j++)                                       \
          for (int i = 1; i < nx - 1; i++) {                                   \
            int64_t o = IDX3(i, j, k, nx, ny);                                 \
            REAL s0 = a0[o] * HP(i, j, k + 1) + a1[o] * HP(i, j + 1, k) +      \
                      a2[o] * HP(i + 1, j, k) +                                \
                      b0[o] * (HP(i, j + 1, k + 1) - HP(i, j - 1, k + 1) -     \
                               HP(i, j + 1, k - 1) + HP(i, j - 1, k - 1)) +    \
                      b1[o] * (HP(i + 1, j + 1, k) - HP(i + 1, j - 1, k) -     \
                               HP(i - 1, j + 1, k) + HP(i - 1, j - 1, k)) +    \
                      b2[o] * (HP(i + 1, j, k + 1) - HP(i + 1, j, k - 1) -     \
                               HP(i - 1, j, k + 1) + HP(i - 1, j, k - 1)) +    \
                      c0[o] * HP(i, j, k - 1) + c1[o] * HP(i, j - 1, k) +      \
                      c2[o] * HP(i - 1, j, k) + wrk1[o];                       \
            REAL ss = (s0 * a3[o] - HP(i, j, k)) * bnd[o];                     \
            REAL v = HP(i, j, k) + omega * ss;                                 \
            dst[o] = v;                                                        \
            double q = (double)ss * (double)ss;                                \
            double t = g + q;                                                  \
            if (fabs(g) >= fabs(q)) gc += (g - t) + q; else gc += (q - t) + g; \
            g = t;                                                             \
          }                                                                    \
      if (gosa) gosa[it] = g + gc;                                             \
      REAL *t = src;                                                           \
      src = dst;                                                               \
      dst = t;                                                                 \
    }                                                                          \
    /* After an even number of sweeps the result is back in p0 (as in the    \
       reference's PSStencilRun(map(p0->p1), map(p1->p0), nn/2)). */         \
  }
#define HP(i, j, k) src[IDX3(i, j, k, nx, ny)]
DEFINE_HIMENO(orc_himeno_f32, float)
DEFINE_HIMENO(orc_himeno_f64, double)
#undef HP

/* ------------------------------------------------------------------------ */
/* Generic flat linear stencil (the descriptor of physis_b200.h).            */
/* Each access follows the reference's per-access index forms:               */
/*  NONE: x + off; PERIODIC: (x + off + n) % n (physis_ref.h:68-79);         */
/*  CLAMP: the conditional get "(x==0) ? c : g(x-1)" generalised to          */
/*  min(max(x + off, 0), n - 1) (test_7-pt-neumann-cond.c:26-32).             */
/* ------------------------------------------------------------------------ */
typedef struct {
  void *data;
  int type;
  int ndims;
  int dims[3];
} orc_grid;

static int64_t orc_index(const psb_generic_stencil *d, const orc_grid *g,
                         int slot, const psb_factor *f, const int *p) {
  int64_t off = 0, stride = 1;
  for (int k = 0; k < g->ndims; k++) {
    int ax = d->grid_axes[slot][k];
    int n = g->dims[k];
    int i = p[ax] + f->offset[ax];
    if (f->boundary == PSB_BOUNDARY_PERIODIC) {
      i = (i + n) % n;
    } else if (f->boundary == PSB_BOUNDARY_CLAMP) {
      i = i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
    }
    off += (int64_t)i * stride;
    stride *= n;
  }
  return off;
}

#define DEFINE_FACTOR(NAME, ACC)                                               \
  static ACC NAME(const psb_generic_stencil *d, const orc_grid *gs,            \
                  const psb_factor *f, const int *p) {                         \
    if (f->grid < 0) return (ACC)f->constant;                                  \
    const orc_grid *g = &gs[f->grid];                                          \
    int64_t o = orc_index(d, g, f->grid, f, p);                                \
    switch (g->type) {                                                         \
      case PS_FLOAT: return (ACC)((const float *)g->data)[o];                  \
      case PS_DOUBLE: return (ACC)((const double *)g->data)[o];                \
      case PS_INT: return (ACC)((const int32_t *)g->data)[o];                  \
      default: return (ACC)((const int64_t *)g->data)[o];                      \
    }                                                                          \
  }
DEFINE_FACTOR(orc_factor_f32, float)
DEFINE_FACTOR(orc_factor_f64, double)
DEFINE_FACTOR(orc_factor_i32, int32_t)
DEFINE_FACTOR(orc_factor_i64, int64_t)

static void orc_store(orc_grid *g, int64_t o, double vd, int64_t vi, int isint,
                      float vf, int isf) {
  switch (g->type) {
    case PS_FLOAT: ((float *)g->data)[o] = isf ? vf : (isint ? (float)vi : (float)vd); break;
    case PS_DOUBLE: ((double *)g->data)[o] = isf ? (double)vf : (isint ? (double)vi : vd); break;
    case PS_INT: ((int32_t *)g->data)[o] = isf ? (int32_t)vf : (isint ? (int32_t)vi : (int32_t)vd); break;
    default: ((int64_t *)g->data)[o] = isf ? (int64_t)vf : (isint ? vi : (int64_t)vd); break;
  }
}

/* One application of the stencil over dom [lo, hi). color: -1 for all
 * points, 0 red / 1 black for red-black maps: a point is visited when
 * (x + y + z + color) is even, which is the x start
 * lo0 + ((lo0 & 1) ^ (y + z + color) % 2) of test_redblack.manual.ref.c:13
 * for the domains the tests use. */
void orc_generic_apply(const psb_generic_stencil *d, void *const *datas,
                       const int *dims_flat, const int *lo, const int *hi,
                       int color) {
  orc_grid gs[PSB_MAX_GRIDS];
  for (int i = 0; i < d->ngrids; i++) {
    gs[i].data = datas[i];
    gs[i].type = d->grid_type[i];
    gs[i].ndims = 0;
    for (int k = 0; k < 3; k++) {
      gs[i].dims[k] = dims_flat[i * 3 + k];
      if (d->grid_axes[i][k] >= 0) gs[i].ndims = k + 1;
    }
  }
  int lo3[3] = {0, 0, 0}, hi3[3] = {1, 1, 1};
  for (int k = 0; k < d->ndims; k++) {
    lo3[k] = lo[k];
    hi3[k] = hi[k];
  }
  orc_grid *out = &gs[d->out_grid];
  psb_factor self;
  memset(&self, 0, sizeof(self));
  for (int z = lo3[2]; z < hi3[2]; z++)
    for (int y = lo3[1]; y < hi3[1]; y++)
      for (int x = lo3[0]; x < hi3[0]; x++) {
        int p[3] = {x, y, z};
        if (color >= 0 && ((x + y + z + color) & 1)) continue;
        int64_t o = orc_index(d, out, d->out_grid, &self, p);
        switch (d->accum_type) {
          case PS_FLOAT: {
            float acc = 0;
            for (int t = 0; t < d->nterms; t++) {
              float v = orc_factor_f32(d, gs, &d->terms[t].a, p) *
                        orc_factor_f32(d, gs, &d->terms[t].b, p);
              acc = t ? acc + v : v;
            }
            if (d->has_post) acc = acc * orc_factor_f32(d, gs, &d->post, p);
            orc_store(out, o, 0, 0, 0, acc, 1);
            break;
          }
          case PS_DOUBLE: {
            double acc = 0;
            for (int t = 0; t < d->nterms; t++) {
              double v = orc_factor_f64(d, gs, &d->terms[t].a, p) *
                         orc_factor_f64(d, gs, &d->terms[t].b, p);
              acc = t ? acc + v : v;
            }
            if (d->has_post) acc = acc * orc_factor_f64(d, gs, &d->post, p);
            orc_store(out, o, acc, 0, 0, 0, 0);
            break;
          }
          case PS_INT: {
            int32_t acc = 0;
            for (int t = 0; t < d->nterms; t++) {
              int32_t v = orc_factor_i32(d, gs, &d->terms[t].a, p) *
                          orc_factor_i32(d, gs, &d->terms[t].b, p);
              acc = t ? acc + v : v;
            }
            if (d->has_post) acc = acc * orc_factor_i32(d, gs, &d->post, p);
            orc_store(out, o, 0, acc, 1, 0, 0);
            break;
          }
          default: {
            int64_t acc = 0;
            for (int t = 0; t < d->nterms; t++) {
              int64_t v = orc_factor_i64(d, gs, &d->terms[t].a, p) *
                          orc_factor_i64(d, gs, &d->terms[t].b, p);
              acc = t ? acc + v : v;
            }
            if (d->has_post) acc = acc * orc_factor_i64(d, gs, &d->post, p);
            orc_store(out, o, 0, acc, 1, 0, 0);
            break;
          }
        }
      }
}

/* ------------------------------------------------------------------------ */
/* Reductions                                                                */
/* ------------------------------------------------------------------------ */
/* The reference CPU fold (libphysis_rt_ref.cc:26-37, reduce.h:19-55). */
void orc_fold_f32(int op, const float *d, int64_t n, float *out) {
  float v = d[0];
  for (int64_t i = 1; i < n; i++) {
    float x = d[i];
    switch (op) {
      case PS_MAX: v = (v > x) ? v : x; break;
      case PS_MIN: v = (v < x) ? v : x; break;
      case PS_SUM: v = v + x; break;
      default: v = v * x; break;
    }
  }
  *out = v;
}
void orc_fold_f64(int op, const double *d, int64_t n, double *out) {
  double v = d[0];
  for (int64_t i = 1; i < n; i++) {
    double x = d[i];
    switch (op) {
      case PS_MAX: v = (v > x) ? v : x; break;
      case PS_MIN: v = (v < x) ? v : x; break;
      case PS_SUM: v = v + x; break;
      default: v = v * x; break;
    }
  }
  *out = v;
}
/* Exact-as-possible FP64 reference values used to bound the GPU reduction:
 * sum with Neumaier compensation, product in FP64, and sum of |x_i| for the
 * error bound gamma_n * sum|x_i|. */
void orc_sum_f64(const void *d, int type, int64_t n, double *sum, double *abssum) {
  double s = 0, c = 0, a = 0;
  for (int64_t i = 0; i < n; i++) {
    double x = type == PS_FLOAT ? (double)((const float *)d)[i] : ((const double *)d)[i];
    double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
    a += fabs(x);
  }
  *sum = s + c;
  *abssum = a;
}
