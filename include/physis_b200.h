/*
 * physis_b200.h -- C ABI of the B200-native runtime for the Physis stencil DSL.
 *
 * Two groups of entry points live here:
 *
 *  1. The drop-in boundary: the exact symbols, types and macros that code
 *     generated by the Physis CUDA target (and a user's main) link against.
 *     Their signatures and struct layouts follow the reference headers
 *     include/physis/physis_cuda.h:18-150,234-238 and
 *     include/physis/physis_common.h:28-150 so that a generated
 *     <file>.cuda.cu compiles and links unchanged against this library
 *     instead of libphysis_rt_cuda.
 *
 *  2. Translator-free and native extensions (prefix psb_ / PSGrid*New /
 *     PSStencil*): the user API of include/physis/physis_user.h:52-114 made
 *     callable without the ROSE translator (stencils are named by a
 *     descriptor instead of a C function), plus status-returning entry
 *     points for stencil descriptors, runs, reductions, batching and serving.
 *
 * Every function in group 1 returns void like the reference and reports CUDA
 * failures the way the reference does (message on stderr, exit(EXIT_FAILURE)),
 * see runtime/runtime_common_cuda.h:16-23. Group-2 functions return a
 * psb_status instead and never exit; PSGetLastError() reads the last status.
 *
 * All device memory is on one GPU (device 0 unless PHYSIS_B200_DEVICE is set).
 */
#ifndef PHYSIS_B200_H_
#define PHYSIS_B200_H_

#include <stdint.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Common types (include/physis/physis_common.h:44-101, types.h:17-23,       */
/* reduce.h:16-21)                                                            */
/* ------------------------------------------------------------------------ */

#define PS_MAX_DIM (3)
typedef int32_t PSIndex;                 /* physis_common.h:44 (32-bit index) */
typedef int PSVectorInt[PS_MAX_DIM];     /* physis_common.h:61 */
typedef PSVectorInt PSPoint;

typedef int PSType;
enum PSPrimitiveType {                   /* types.h:17-23 */
  PS_INT = 0,
  PS_LONG = 1,
  PS_FLOAT = 2,
  PS_DOUBLE = 3,
  PS_USER = 4
};

enum PSReduceOp {                        /* reduce.h:16-21 */
  PS_MAX,
  PS_MIN,
  PS_SUM,
  PS_PROD
};

typedef struct {                         /* physis_common.h:86-91 */
  PSIndex min[PS_MAX_DIM];
  PSIndex max[PS_MAX_DIM];
  PSIndex local_min[PS_MAX_DIM];
  PSIndex local_max[PS_MAX_DIM];
} __PSDomain;
typedef __PSDomain PSDomain1D;
typedef __PSDomain PSDomain2D;
typedef __PSDomain PSDomain3D;

#define INVALID_GRID (NULL)

/* ------------------------------------------------------------------------ */
/* Device grid structs passed by value into generated kernels               */
/* (physis_cuda.h:18-97). Layout: int dim[N] then the element pointer.       */
/* ------------------------------------------------------------------------ */

typedef struct { int dim[1]; void *p0; } __PSGrid1D_dev;
typedef struct { int dim[1]; float *p0; } __PSGrid1DFloat_dev;
typedef struct { int dim[1]; double *p0; } __PSGrid1DDouble_dev;
typedef struct { int dim[1]; int *p0; } __PSGrid1DInt_dev;
typedef struct { int dim[1]; long *p0; } __PSGrid1DLong_dev;
typedef struct { int dim[2]; void *p0; } __PSGrid2D_dev;
typedef struct { int dim[2]; float *p0; } __PSGrid2DFloat_dev;
typedef struct { int dim[2]; double *p0; } __PSGrid2DDouble_dev;
typedef struct { int dim[2]; int *p0; } __PSGrid2DInt_dev;
typedef struct { int dim[2]; long *p0; } __PSGrid2DLong_dev;
typedef struct { int dim[3]; void *p0; } __PSGrid3D_dev;
typedef struct { int dim[3]; float *p0; } __PSGrid3DFloat_dev;
typedef struct { int dim[3]; double *p0; } __PSGrid3DDouble_dev;
typedef struct { int dim[3]; int *p0; } __PSGrid3DInt_dev;
typedef struct { int dim[3]; long *p0; } __PSGrid3DLong_dev;
typedef struct { int dim[3]; void *p0; } __PSGrid_dev;

/* Host grid descriptor (physis_cuda.h:99-106). For grids created through
 * __PSGridNew, p0 and dev->p0 point at a dense x-fastest array exactly like
 * the reference. For grids created through PSGrid{1,2,3}D*New (the
 * translator-free API) the device array is pitched with a resident halo;
 * p0 then points at logical element (0,0,0) and psb_grid_layout() gives
 * the strides. Either kind is accepted by every entry point below. */
typedef struct {
  void *p0;
  PSVectorInt dim;
  int elm_size;
  int num_dims;
  int64_t num_elms;
  __PSGrid_dev *dev;
} __PSGrid;

typedef __PSGrid *PSGrid1DFloat;
typedef __PSGrid *PSGrid2DFloat;
typedef __PSGrid *PSGrid3DFloat;
typedef __PSGrid *PSGrid1DDouble;
typedef __PSGrid *PSGrid2DDouble;
typedef __PSGrid *PSGrid3DDouble;
typedef __PSGrid *PSGrid1DInt;
typedef __PSGrid *PSGrid2DInt;
typedef __PSGrid *PSGrid3DInt;
typedef __PSGrid *PSGrid1DLong;
typedef __PSGrid *PSGrid2DLong;
typedef __PSGrid *PSGrid3DLong;
#define DeclareGrid1D(name, type) typedef __PSGrid *PSGrid1D##name;
#define DeclareGrid2D(name, type) typedef __PSGrid *PSGrid2D##name;
#define DeclareGrid3D(name, type) typedef __PSGrid *PSGrid3D##name;
#define PSGridDim(p, d) ((p)->dim[(d)])           /* physis_cuda.h:125 */
#define __PSGridDimDev(p, d) ((p)->dim[d])

/* Dense offset helpers used by generated code (physis_cuda.h:158-231):
 * x-fastest linear offsets, and the periodic form that wraps each index
 * with (i + n) % n. They apply to grids made by __PSGridNew (dense). */
#if defined(__CUDACC__)
#define PSB_HD __host__ __device__
#else
#define PSB_HD
#endif
static inline PSB_HD PSIndex __PSB_Off3(const int *d, PSIndex i, PSIndex j, PSIndex k) {
  return i + j * d[0] + k * d[0] * d[1];
}
static inline PSB_HD PSIndex __PSB_Wrap(PSIndex i, int n) { return (i + n) % n; }
static inline PSIndex __PSGridGetOffset1D(__PSGrid *g, PSIndex i1) { (void)g; return i1; }
static inline PSIndex __PSGridGetOffset2D(__PSGrid *g, PSIndex i1, PSIndex i2) {
  return i1 + i2 * g->dim[0];
}
static inline PSIndex __PSGridGetOffset3D(__PSGrid *g, PSIndex i1, PSIndex i2, PSIndex i3) {
  return __PSB_Off3(g->dim, i1, i2, i3);
}
static inline PSIndex __PSGridGetOffsetPeriodic1D(__PSGrid *g, PSIndex i1) {
  return __PSB_Wrap(i1, g->dim[0]);
}
static inline PSIndex __PSGridGetOffsetPeriodic2D(__PSGrid *g, PSIndex i1, PSIndex i2) {
  return __PSB_Wrap(i1, g->dim[0]) + __PSB_Wrap(i2, g->dim[1]) * g->dim[0];
}
static inline PSIndex __PSGridGetOffsetPeriodic3D(__PSGrid *g, PSIndex i1, PSIndex i2,
                                                  PSIndex i3) {
  return __PSB_Off3(g->dim, __PSB_Wrap(i1, g->dim[0]), __PSB_Wrap(i2, g->dim[1]),
                    __PSB_Wrap(i3, g->dim[2]));
}
#if defined(__CUDACC__)
static inline __device__ PSIndex __PSGridGetOffset1DDev(const void *g, PSIndex i1) {
  (void)g;
  return i1;
}
static inline __device__ PSIndex __PSGridGetOffset2DDev(const void *g, PSIndex i1, PSIndex i2) {
  return i1 + i2 * ((const __PSGrid_dev *)g)->dim[0];
}
static inline __device__ PSIndex __PSGridGetOffset3DDev(const void *g, PSIndex i1, PSIndex i2,
                                                        PSIndex i3) {
  return __PSB_Off3(((const __PSGrid_dev *)g)->dim, i1, i2, i3);
}
static inline __device__ PSIndex __PSGridGetOffsetPeriodic1DDev(const void *g, PSIndex i1) {
  return __PSB_Wrap(i1, ((const __PSGrid_dev *)g)->dim[0]);
}
static inline __device__ PSIndex __PSGridGetOffsetPeriodic2DDev(const void *g, PSIndex i1,
                                                               PSIndex i2) {
  const int *d = ((const __PSGrid_dev *)g)->dim;
  return __PSB_Wrap(i1, d[0]) + __PSB_Wrap(i2, d[1]) * d[0];
}
static inline __device__ PSIndex __PSGridGetOffsetPeriodic3DDev(const void *g, PSIndex i1,
                                                               PSIndex i2, PSIndex i3) {
  const int *d = ((const __PSGrid_dev *)g)->dim;
  return __PSB_Off3(d, __PSB_Wrap(i1, d[0]), __PSB_Wrap(i2, d[1]), __PSB_Wrap(i3, d[2]));
}
#endif

typedef void *(*__PSGrid_devNewFunc)(int num_dims, PSVectorInt dim);
typedef void (*__PSGrid_devFreeFunc)(void *);
typedef void (*__PSGrid_devCopyinFunc)(void *g, const void *src);
typedef void (*__PSGrid_devCopyoutFunc)(void *g, void *dst);

/* ------------------------------------------------------------------------ */
/* Group 1: drop-in ABI (libphysis_rt_cuda.cc:28-191, reduce_cuda.cu:21-29,  */
/* runtime_common.cc:13-50)                                                  */
/* ------------------------------------------------------------------------ */

/* Replaces PSInit (libphysis_rt_cuda.cc:28-39). Parses and removes
 * --physis-trace (runtime/runtime.cc:81-91), selects the GPU, checks it is
 * sm_100, creates the runtime stream. Varargs: the grid extents, ignored. */
void PSInit(int *argc, char ***argv, int grid_num_dims, ...);
/* Replaces PSFinalize (libphysis_rt_cuda.cc:41-44). */
void PSFinalize(void);
/* Replaces __PSGridNew (libphysis_rt_cuda.cc:51-102): dense, zeroed device
 * array; func != NULL delegates to the user-type allocator like the
 * reference. Returns INVALID_GRID if the allocation fails. */
__PSGrid *__PSGridNew(int elm_size, int num_dims, PSVectorInt dim,
                      __PSGrid_devNewFunc func);
/* Replaces __PSGridFree (libphysis_rt_cuda.cc:104-114). Also releases the
 * host descriptor, which the reference leaks. */
void __PSGridFree(__PSGrid *g, __PSGrid_devFreeFunc func);
/* Replace __PSGridCopyin/__PSGridCopyout (libphysis_rt_cuda.cc:116-139):
 * whole-grid copy from/to a dense x-fastest host array; returns when done. */
void __PSGridCopyin(void *g, const void *src_array, __PSGrid_devCopyinFunc func);
void __PSGridCopyout(void *g, void *dst_array, __PSGrid_devCopyoutFunc func);
/* No-ops like the reference (libphysis_rt_cuda.cc:141-142). */
void __PSGridSwap(__PSGrid *g);
void __PSGridMirror(__PSGrid *g);
/* Replaces __PSGridGetID (libphysis_rt_cuda.cc:47-49): always 0. */
int __PSGridGetID(__PSGrid *g);
/* Replaces __PSGridSet (libphysis_rt_cuda.cc:164-179): varargs are one
 * PSIndex per dimension; writes one element from buf. */
void __PSGridSet(__PSGrid *g, void *buf, ...);
/* Reads one element into buf (counterpart of __PSGridSet; physis_ref.h:53). */
void __PSGridGet(__PSGrid *g, void *buf, ...);
/* Replace PSDomain{1,2,3}DNew (libphysis_rt_cuda.cc:144-162). */
PSDomain1D PSDomain1DNew(PSIndex minx, PSIndex maxx);
PSDomain2D PSDomain2DNew(PSIndex minx, PSIndex maxx, PSIndex miny, PSIndex maxy);
PSDomain3D PSDomain3DNew(PSIndex minx, PSIndex maxx, PSIndex miny, PSIndex maxy,
                         PSIndex minz, PSIndex maxz);
/* Replace __PSReduceGridFloat/Double (reduce_cuda.cu:21-29): reduce every
 * element of the grid (num_elms, not a domain) with op into *buf. SUM and
 * PROD accumulate in FP64 (Neumaier-compensated for double grids) in a fixed
 * order, so results are deterministic run to run. */
void __PSReduceGridFloat(void *buf, enum PSReduceOp op, __PSGrid *g);
void __PSReduceGridDouble(void *buf, enum PSReduceOp op, __PSGrid *g);
/* Replaces __PSCheckCudaError (libphysis_rt_cuda.cc:185-191). */
void __PSCheckCudaError(const char *message);
/* Replaces __PSRandomInit (runtime_common.cc:35-50): a shuffled 0..n-1. */
void *__PSRandomInit(int n);
/* Trace stream, set by --physis-trace (runtime_common.cc:13). */
extern FILE *__ps_trace;

/* ------------------------------------------------------------------------ */
/* Group 2a: translator-free user API (physis_user.h:52-114,                */
/* physis_common.h:81-84)                                                    */
/* ------------------------------------------------------------------------ */

/* Grid constructors declared by DeclareGrid{1,2,3}D (physis_user.h:52-75).
 * The trailing varargs of the reference (grid attributes) are ignored.
 * These create pitched grids: rows padded to 128 bytes, logical x = 0 on a
 * 128-byte boundary, and a resident halo of PSB_HALO cells in every
 * dimension that the runtime keeps consistent for periodic reads. */
PSGrid1DFloat PSGrid1DFloatNew(PSIndex nx, ...);
PSGrid2DFloat PSGrid2DFloatNew(PSIndex nx, PSIndex ny, ...);
PSGrid3DFloat PSGrid3DFloatNew(PSIndex nx, PSIndex ny, PSIndex nz, ...);
PSGrid1DDouble PSGrid1DDoubleNew(PSIndex nx, ...);
PSGrid2DDouble PSGrid2DDoubleNew(PSIndex nx, PSIndex ny, ...);
PSGrid3DDouble PSGrid3DDoubleNew(PSIndex nx, PSIndex ny, PSIndex nz, ...);
PSGrid1DInt PSGrid1DIntNew(PSIndex nx, ...);
PSGrid2DInt PSGrid2DIntNew(PSIndex nx, PSIndex ny, ...);
PSGrid3DInt PSGrid3DIntNew(PSIndex nx, PSIndex ny, PSIndex nz, ...);
PSGrid1DLong PSGrid1DLongNew(PSIndex nx, ...);
PSGrid2DLong PSGrid2DLongNew(PSIndex nx, PSIndex ny, ...);
PSGrid3DLong PSGrid3DLongNew(PSIndex nx, PSIndex ny, PSIndex nz, ...);
void PSGridCopyin(void *g, const void *src_array);   /* physis_common.h:81 */
void PSGridCopyout(void *g, void *dst_array);        /* physis_common.h:82 */
void PSGridFree(void *g);                            /* physis_common.h:84 */

/* A stencil is named by a kernel id (psb_kernel) where the reference passes
 * a C function. PSStencilMap(k, dom, grids..., scalars...) binds it, like
 * physis_user.h:104-106; scalars are passed as C varargs (float promotes to
 * double). PSStencilRun(m0, m1, ..., iter) runs the maps in order iter
 * times (physis_user.h:112); the macro counts the arguments so a trailing
 * iteration count is optional, as in the reference. PSReduce(&v, op, g)
 * reduces a grid (physis_user.h:114, docs/programming.md:283). */
typedef int PSStencil;
PSStencil __PSStencilMap(void *kernel, ...);
PSStencil __PSStencilMapRedBlack(void *kernel, ...);
PSStencil __PSStencilMapRed(void *kernel, ...);
PSStencil __PSStencilMapBlack(void *kernel, ...);
void __PSStencilRunN(int nargs, ...);
void PSReduce(void *v, ...);
/* PSReduce(&v, op, kernel, dom, grids...): the kernel-function form of
 * docs/programming.md:298-320 (not implemented by the reference,
 * translator/reference_translator.cc:1357-1360). kernel is a registered
 * generic stencil; the value it would emit at each point of dom (in the
 * emitted grid's element type, which v also has) is reduced by op, and
 * nothing is stored. The PSReduce macro below dispatches both forms on the
 * argument count. */
void __PSReduceN(int nargs, void *v, ...);

#define PSB__NARGS_(_1,_2,_3,_4,_5,_6,_7,_8,_9,_10,_11,_12,_13,_14,_15,_16,N,...) N
#define PSB__NARGS(...) PSB__NARGS_(__VA_ARGS__,16,15,14,13,12,11,10,9,8,7,6,5,4,3,2,1)
#define PSStencilMap(k, ...) __PSStencilMap((void *)(intptr_t)(k), __VA_ARGS__)
#define PSStencilMapRedBlack(k, ...) __PSStencilMapRedBlack((void *)(intptr_t)(k), __VA_ARGS__)
#define PSStencilMapRed(k, ...) __PSStencilMapRed((void *)(intptr_t)(k), __VA_ARGS__)
#define PSStencilMapBlack(k, ...) __PSStencilMapBlack((void *)(intptr_t)(k), __VA_ARGS__)
#define PSStencilRun(...) __PSStencilRunN(PSB__NARGS(__VA_ARGS__), __VA_ARGS__)
#define PSReduce(...) __PSReduceN(PSB__NARGS(__VA_ARGS__), __VA_ARGS__)

/* ------------------------------------------------------------------------ */
/* Group 2b: native status-returning API                                    */
/* ------------------------------------------------------------------------ */

typedef enum {
  PSB_OK = 0,
  PSB_ERR_INVALID = 1,        /* bad argument, shape or descriptor */
  PSB_ERR_NOMEM = 2,          /* device allocation or budget exceeded */
  PSB_ERR_CUDA = 3,           /* a CUDA call failed */
  PSB_ERR_NOT_INIT = 4,       /* PSInit / psb_init not called */
  PSB_ERR_TIMEOUT = 5,        /* a bounded device-side wait gave up */
  PSB_ERR_UNSUPPORTED = 6,    /* valid request this build does not run */
  PSB_ERR_CANCELLED = 7,      /* a serving request was cancelled */
  PSB_ERR_BUSY = 8,           /* queue full / resource in use */
  PSB_ERR_BOUNDS = 9          /* a compiled stencil read outside its grid
                                 (the read returned 0, nothing was touched) */
} psb_status;

/* Halo (ghost) width of pitched grids, in cells, in y and z. In x the halo
 * is one 128-byte line on the left and at least PSB_HALO cells on the right. */
#define PSB_HALO 2
#define PSB_MAX_GRIDS 16
#define PSB_MAX_TERMS 32
#define PSB_MAX_PARAMS 16
#define PSB_B200_MAX_RUN_MAPS 16

typedef enum {
  PSB_LAYOUT_DENSE = 0,       /* x-fastest, no padding (reference layout) */
  PSB_LAYOUT_PITCHED = 1      /* 128-byte rows, resident halo */
} psb_layout;

/* Built-in kernels usable as the first argument of PSStencilMap. Ids of
 * generic descriptors registered with psb_generic_register follow. */
typedef enum {
  /* 7-point diffusion, examples/diffusion-benchmark/diffusion3d_physis.c:29-58:
   * grids (in, out); scalars (ce, cw, cn, cs, ct, cb, cc); out =
   * cc*c + cw*w + ce*e + cs*s + cn*n + cb*b + ct*t, neighbours clamped at
   * the grid faces. Element type from the grids (float or double). */
  PSB_KERNEL_DIFFUSION7 = 1,
  /* The same update with periodic neighbours (PSGridGetPeriodic). */
  PSB_KERNEL_DIFFUSION7_PERIODIC = 2,
  /* 19-point Himeno Jacobi, examples/himeno/himenobmtxpa_physis.c:331-361:
   * grids (p_in, p_out, a0, a1, a2, a3, b0, b1, b2, c0, c1, c2, bnd, wrk1);
   * scalar omega. float only. */
  PSB_KERNEL_HIMENO19 = 3,
  PSB_KERNEL_FIRST_GENERIC = 64,
  /* Ids of compiled stencils (psb_compiled_register) start here. */
  PSB_KERNEL_FIRST_COMPILED = 1 << 16
} psb_kernel;

/* Per-access boundary handling of a generic term (reference forms:
 * PSGridGet / PSGridGetPeriodic / the clamped conditional get of
 * test_7-pt-neumann-cond.c:26-32). */
typedef enum {
  PSB_BOUNDARY_NONE = 0,      /* caller keeps every access inside the grid */
  PSB_BOUNDARY_PERIODIC = 1,  /* index wraps: (i + n) % n per axis */
  PSB_BOUNDARY_CLAMP = 2      /* index clamps to [0, n-1] per axis */
} psb_boundary;

/* One factor of a generic term: a grid read at the point plus offset, or a
 * constant when grid < 0. axes[d] names the domain axis (0..2) that grid
 * dimension d follows, which lets a 1-D or 2-D grid be read inside a 3-D
 * stencil (test_mixed-dim*.c); -1 ends the list. */
typedef struct {
  int grid;
  int offset[3];
  int boundary;
  double constant;
} psb_factor;

typedef struct {
  psb_factor a;
  psb_factor b;
} psb_term;

/* A flat linear stencil: out(p) = post(p) * (t0 + t1 + ... + t{n-1}) where
 * ti = a_i * b_i, both factors converted to accum_type first, summed left
 * to right in accum_type (the order C evaluates a + b + c). If has_post is
 * 0 the multiply is skipped. The result is converted to the out grid's
 * type. Grid slots 0..ngrids-1 are bound by PSStencilMap in order. */
typedef struct {
  int ndims;                          /* dimensionality of the domain */
  int ngrids;
  int grid_type[PSB_MAX_GRIDS];       /* PS_FLOAT / PS_DOUBLE / PS_INT / PS_LONG */
  int grid_axes[PSB_MAX_GRIDS][3];
  int out_grid;                       /* slot that is emitted */
  int accum_type;
  int nterms;
  psb_term terms[PSB_MAX_TERMS];
  int has_post;
  psb_factor post;
  int redblack;                       /* 0: all points; set by the map call */
} psb_generic_stencil;

/* Initialise without argc/argv (same effect as PSInit). */
psb_status psb_init(void);
psb_status PSGetLastError(void);
const char *psb_status_string(psb_status s);

/* Grid creation with an explicit layout and element type (PSPrimitiveType).
 * dims has num_dims entries. */
/* Grids of user-defined point types (the reference's DeclareGrid3D(Name,
 * struct T) with struct members, physis_user.h:52-75, tests
 * test_user-defined-type-*.c; its CUDA target keeps them as SoA device
 * arrays, translator/cuda_runtime_builder.cc:319-1100). A type is a list of
 * fields, each `count` scalars of one primitive type at `offset` bytes into
 * a record of record_bytes. On the device every scalar component (field f,
 * element k) is its own pitched grid; copy-in/copy-out of the user-type
 * grid (PSGridCopyin/Copyout, psb_grid_copyin/copyout_async) convert between
 * the host array of records and the components on the device. Stencils bind
 * components (psb_grid_component) like ordinary grids. */
#define PSB_MAX_FIELDS 16
#define PSB_MAX_COMPONENTS 64
typedef struct {
  int nfields;
  size_t record_bytes;
  int field_type[PSB_MAX_FIELDS];     /* PS_FLOAT / PS_DOUBLE / PS_INT / PS_LONG */
  int field_count[PSB_MAX_FIELDS];    /* scalars in the field (array members) */
  size_t field_offset[PSB_MAX_FIELDS];
} psb_user_type;
psb_status psb_grid_new_user(int num_dims, const PSIndex *dims, const psb_user_type *type,
                             __PSGrid **out);
/* Component k of field f of a user-type grid: a grid handle sharing the
 * component's storage (valid until the user-type grid is freed; do not
 * free it). */
psb_status psb_grid_component(__PSGrid *g, int field, int index, __PSGrid **out);
psb_status psb_grid_new(int type, int num_dims, const PSIndex *dims, int layout,
                        __PSGrid **out);
/* Strides in elements between y rows and z planes, the layout and the
 * allocation size in bytes. */
psb_status psb_grid_layout(const __PSGrid *g, int64_t *stride_y, int64_t *stride_z,
                           int *layout, int64_t *alloc_bytes);
/* Asynchronous copies on the runtime stream (host buffers should be pinned
 * for overlap; see psb_host_alloc). psb_sync waits for the stream. */
psb_status psb_grid_copyin_async(__PSGrid *g, const void *src);
psb_status psb_grid_copyout_async(__PSGrid *g, void *dst);
psb_status psb_sync(void);
psb_status psb_host_alloc(size_t bytes, void **ptr);
psb_status psb_host_free(void *ptr);
/* Fill a grid's interior on the device with a seeded synthetic field (no
 * counterpart in the reference; used by benchmarks and tests). Element i =
 * x + nx*(y + ny*z) gets h = splitmix64(seed*0x9E3779B97F4A7C15 + i) and
 * kind 0: lo + (hi-lo) * (h >> 40) * 2^-24; kind 1: lo; kind 2: 1 inside and
 * 0 on the faces; kind 3: (z/(nz-1))^2 -- computed in double, rounded once.
 * Asynchronous on the runtime stream. */
psb_status psb_grid_fill(__PSGrid *g, int kind, uint64_t seed, double lo, double hi);
/* Copy one grid's interior into another grid of the same shape and type. */
psb_status psb_grid_copy(__PSGrid *dst, const __PSGrid *src);

/* Register a generic stencil; *kernel_id is usable with PSStencilMap. */
psb_status psb_generic_register(const psb_generic_stencil *desc, int *kernel_id);
/* Which kernel ran the last application of a generic stencil (no
 * counterpart in the reference): PSB_IMPL_TMA for the TMA z-streaming
 * kernel (3-D, float or double, every grid read of the accumulation type
 * with offsets within +-2, at most four grids read, not in place, not
 * red-black), PSB_IMPL_GENERIC for the thread-per-point kernel, which runs
 * every other form and every map under psb_set_impl(PSB_IMPL_PLAIN or
 * PSB_IMPL_GENERIC). */
psb_status psb_generic_last_impl(int *impl);
/* Whether the last TMA application of a generic stencil ran a kernel
 * compiled at run time for its table (1) or the kernel that interprets the
 * table (0). Tables on the TMA path are compiled by NVRTC for sm_100a when
 * the map first runs --
 * the reference's translator likewise emits one kernel per stencil
 * (translator/cuda_translator.cc:615-869) -- and cached per process for
 * every table of the same shape (coefficients are launch arguments). Same
 * arithmetic, same results; without NVRTC or the library's device headers
 * (csrc/ beside lib/, or $PHYSIS_B200_CSRC) the interpreting kernel runs. */
psb_status psb_generic_last_compiled(int *compiled);
/* Run-time compilation of generic tables on (1, the default unless
 * $PHYSIS_B200_GENERIC_COMPILE=0) or off (0). */
psb_status psb_set_generic_compile(int on);

/* Compiled stencils: a DSL stencil function (docs/programming.md:117-190 of
 * the reference: `const int` index parameters, grids, scalars;
 * PSGridGet / PSGridGetPeriodic / PSGridEmit / PSGridEmitUtype / PSGridDim)
 * translated by the front end physis_b200/dsl.py into a CUDA kernel of its
 * own shared library, in place of the reference's translator
 * (translator/cuda_translator.cc, which needs ROSE). The library exports a
 * launch function; registering it gives a kernel id usable with
 * PSStencilMap / PSStencilRun like a built-in. At each application the
 * runtime passes the domain, one view per scalar component of the bound
 * grids (a grid of a user-defined point type gives one per component, in
 * field order) and the map's scalars; the kernel runs on the given stream. */
#define PSB_MAX_VIEWS 64
typedef struct {
  void *origin;          /* element (0,0,0) */
  int64_t sy, sz;        /* element strides of y and z */
  int n[3];              /* extents (1 past the grid's dimensions) */
  int type;              /* PSPrimitiveType */
} psb_grid_view;

typedef struct {
  int lo[3], hi[3];      /* domain, half-open; unused dimensions [0, 1) */
  int color;             /* -1 every point; 0 / 1 red / black points */
  int nviews, nparams;
  psb_grid_view views[PSB_MAX_VIEWS];
  double params[PSB_MAX_PARAMS];
  int *error;            /* device word; a read outside its grid sets it to
                            PSB_ERR_BOUNDS (reported by psb_sync / copy-out) */
  int device;            /* CUDA device of the grids and the stream */
} psb_launch_args;

typedef psb_status (*psb_compiled_launch)(const psb_launch_args *args, void *cuda_stream);
/* The staged form of a compiled stencil: its body run over the library's TMA
 * plane ring (the kernel body of the generic TMA path, csrc/k_generic_tma.cuh).
 * The library prepares the tensor maps, table, output view, domain and ring
 * geometry (opaque here; layouts of that header) and the launch shape. */
typedef psb_status (*psb_compiled_staged)(const void *maps, const void *table, const void *out,
                                          const void *domain, const void *geometry, int *error,
                                          unsigned blocks, unsigned shared_bytes,
                                          void *cuda_stream);

typedef struct {
  int ndims;                          /* index parameters of the function */
  int ngrids;                         /* grid parameters */
  int grid_type[PSB_MAX_GRIDS];       /* element type, PS_USER for a point type */
  int grid_ndims[PSB_MAX_GRIDS];
  int grid_components[PSB_MAX_GRIDS]; /* views of the grid: 1, or the point
                                         type's scalar components */
  int nviews;
  int view_type[PSB_MAX_VIEWS];       /* element type of each view */
  int view_emits[PSB_MAX_VIEWS];      /* 1 if the function emits into the view */
  int view_reads_offset[PSB_MAX_VIEWS]; /* 1 if it reads the view off the point */
  int nparams;                        /* scalar parameters after the grids */
  int param_type[PSB_MAX_PARAMS];     /* PS_FLOAT / PS_DOUBLE / PS_INT / PS_LONG
                                         (how PSStencilMap's varargs read them) */
  psb_compiled_launch launch;
  /* Optional staged form (staged != NULL): a 3-D function of one element
   * type (staged_type, PS_FLOAT or PS_DOUBLE) over primitive grids that
   * emits, once and unconditionally, into grid staged_emit (which it does
   * not read) and reads every other grid only at constant offsets within
   * +-2 of the point, between read_lo and read_hi per axis (read_lo > read_hi
   * on axis 0: the grid is not read). The library runs it when the map fits
   * (TMA-ready layouts, no red-black colour, at most four grids read, the
   * emitted grid not bound to a read parameter, and every read range inside
   * its grid over the whole domain) and otherwise calls `launch`.
   * staged_checked (optional, with staged): the same staged form with every
   * read that leaves the point checked against its grid (a read outside
   * reads 0 and sets PSB_ERR_BOUNDS, as `launch` does). The library runs it
   * when a read range may leave its grid over the domain (reads under face
   * tests, e.g. `x == 0 ? c : PSGridGet(g, x-1, y, z)`) and the domain lies
   * inside every grid read.
   * read_periodic[g] = 1: grid g is read with PSGridGetPeriodic (within
   * +-2; read_lo/read_hi cover these reads and any plain ones); the staged
   * forms read its wrapped values from the pitched grid's halo, which the
   * library refreshes first, so they run for such a grid only when it is
   * pitched (PSGrid*New). */
  int staged_type;
  int staged_emit;
  int read_lo[PSB_MAX_GRIDS][3];
  int read_hi[PSB_MAX_GRIDS][3];
  psb_compiled_staged staged;
  psb_compiled_staged staged_checked;
  int read_periodic[PSB_MAX_GRIDS];
} psb_compiled_stencil;

psb_status psb_compiled_register(const psb_compiled_stencil *desc, int *kernel_id);
/* Whether the last application of a compiled stencil ran its staged form
 * (1), the checked staged form (2) or its own thread-per-point launch (0). psb_set_impl(PSB_IMPL_PLAIN or
 * PSB_IMPL_GENERIC) keeps compiled stencils on their own launch. */
psb_status psb_compiled_last_staged(int *staged);

/* Register stencil function `name` of a kernel library made by the front end
 * (which exports psb_dsl_describe_<name>); *status_out gets the status. */
#define PSB_DSL_REGISTER(name, kernel_id_ptr, status_out)            \
  do {                                                                \
    extern void psb_dsl_describe_##name(psb_compiled_stencil *);     \
    psb_compiled_stencil psb_d__;                                     \
    psb_dsl_describe_##name(&psb_d__);                                \
    *(status_out) = psb_compiled_register(&psb_d__, (kernel_id_ptr)); \
  } while (0)

/* Non-varargs map and run. grids: ngrids grid pointers in the kernel's
 * order; params: nparams scalars (converted to the kernel's type). */
psb_status psb_stencil_map(int kernel_id, const __PSDomain *dom, __PSGrid *const *grids,
                           int ngrids, const double *params, int nparams,
                           PSStencil *out);
/* Variant with red-black ordering: color 0 red, 1 black, 2 both in turn
 * (test_redblack*.c; cuda_translator.cc:717-727). */
psb_status psb_stencil_map_rb(int kernel_id, const __PSDomain *dom, __PSGrid *const *grids,
                              int ngrids, const double *params, int nparams, int color,
                              PSStencil *out);
psb_status psb_stencil_run(const PSStencil *maps, int nmaps, int iter);
psb_status psb_stencil_free(PSStencil s);

/* Kernel implementation selected by PSStencilRun for built-in kernels. */
typedef enum {
  PSB_IMPL_AUTO = 0,          /* autotuned fast path (default) */
  PSB_IMPL_PLAIN = 1,         /* one thread per (x,y), z loop, global loads:
                                 the reference's generated-kernel shape */
  PSB_IMPL_TMA = 2,           /* TMA plane pipeline, z-streaming (2.5D) */
  PSB_IMPL_GENERIC = 3        /* the generic term-table kernel */
} psb_impl;
psb_status psb_set_impl(int impl);
/* Arithmetic of the 7-point TMA kernels and of generic tables compiled at
 * run time whose terms are one read times a constant (no counterpart in the
 * reference, whose CUDA target compiles with nvcc's default contraction).
 * PSB_FP_EXACT (default): every product and sum rounded in the reference's
 * term order -- bit-identical to the reference CPU target built without FMA
 * contraction. PSB_FP_FMA: the same term order with each term after the
 * first added by a fused multiply-add (one rounding per term instead of
 * two); for the 7-point kernels within 4 ulp of the exact form per step.
 * Also set by the environment variable PHYSIS_B200_FP_MODE=fma. The plain,
 * Himeno, batched and interpreting generic kernels always use the exact
 * form. */
enum { PSB_FP_EXACT = 0, PSB_FP_FMA = 1 };
psb_status psb_set_fp_mode(int mode);
psb_status psb_get_fp_mode(int *mode);
/* Capture PSStencilRun loops in a CUDA graph (default 1). */
psb_status psb_set_graph(int enable);

/* Himeno residual: sum over the domain of ss*ss in FP64 for each sweep of
 * the given map (ss as in himenobmtxpa_physis.c:356-357), kept in a ring of
 * history_len sweeps (0 disables). One FP64 partial per CTA, combined in a
 * fixed order by the last CTA: no extra pass over memory, no extra launch. */
psb_status psb_himeno_residual_enable(PSStencil map, int history_len);
psb_status psb_himeno_residual(PSStencil map, double *gosa);
/* The last n per-sweep residuals of the map, oldest first (n <= history). */
psb_status psb_himeno_residual_history(PSStencil map, double *out, int n);

/* Reduction of a domain of a grid, FP64 result for every element type. */
psb_status psb_reduce(__PSGrid *g, int op, const __PSDomain *dom, double *result);
/* Kernel-function reduction (the PSReduce kernel form, status-returning):
 * reduce over dom the values generic stencil kernel_id would emit with the
 * given grids (FP64 accumulation, SUM compensated, deterministic). Built-in
 * kernels: PSB_ERR_UNSUPPORTED. */
psb_status psb_reduce_map(int kernel_id, const __PSDomain *dom, __PSGrid *const *grids,
                          int ngrids, const double *params, int nparams, int op,
                          double *result);

/* Allocation-free reduction (no counterpart in the reference). For callers
 * that cannot call cudaMalloc -- a host framework that owns all device memory
 * through its own allocator and budget, or a latency-critical loop where an
 * allocation would synchronise the device -- this reduces a strided device
 * array with the same kernel and order as psb_reduce but keeps its scratch in
 * a fixed static device array of PSB_NOALLOC_SCRATCH_BYTES (held by every GPU
 * that loads the library until exit). It calls no allocator.
 *   data    device pointer to element (0,0,0) of the array
 *   type    PS_FLOAT, PS_DOUBLE, PS_INT or PS_LONG; op a PSReduceOp
 *   extent  nx, ny, nz, each in [1, PSB_NOALLOC_MAX_EXTENT] (else PSB_ERR_INVALID)
 *   stride  elements between rows (>= nx) and between planes (>= stride[0]*ny),
 *           with stride[1] * nz <= INT64_MAX / 8 (else PSB_ERR_INVALID)
 *   stream  a cudaStream_t, or NULL for the legacy default stream; the data
 *           is read in that stream's order, so order it after whatever last
 *           wrote `data` (the runtime works on its own non-blocking stream:
 *           call psb_sync() first when `data` is a runtime grid)
 *   result  host pointer; the call blocks until it is written (FP64 value)
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current: make it before any stream
 * capture. All calls share the array and it keeps the last call's contents;
 * calls that overlap on the GPU race. */
#define PSB_NOALLOC_SCRATCH_BYTES 19200
#define PSB_NOALLOC_MAX_EXTENT 2147483647LL
psb_status psb_reduce_noalloc(const void *data, int type, int op, const int64_t *extent,
                              const int64_t *stride, void *stream, double *result);

/* Timing of the last psb_stencil_run / PSStencilRun: device time (CUDA
 * events on the runtime stream) and the number of kernel launches it
 * issued. */
psb_status psb_last_run_stats(double *device_ms, int64_t *launches);

/* Tile configuration of the fast kernels; the autotuner picks one per
 * (kernel, type, nx, ny, nz) and caches it in a JSON file
 * ($PHYSIS_B200_TUNE_CACHE, default ~/.cache/physis_b200_tune.json). The
 * table measured on B200 (physis_b200/tune_b200.json, beside the library)
 * loads first and the user cache's entries win; PHYSIS_B200_TUNE_SHIPPED=0
 * leaves it out. */
typedef struct {
  int impl;         /* psb_impl */
  int tile_x;       /* points per CTA in x */
  int tile_y;       /* points per CTA in y */
  int z_chunk;      /* planes per CTA work item */
  int stages;       /* pipelined planes in flight */
  int t_depth;      /* temporal blocking depth (1 = none) */
} psb_tune_config;
psb_status psb_autotune(int kernel_id, int type, const PSIndex *dims, int force,
                        psb_tune_config *cfg);
psb_status psb_tune_get(int kernel_id, int type, const PSIndex *dims, psb_tune_config *cfg);
psb_status psb_tune_set(int kernel_id, int type, const PSIndex *dims, const psb_tune_config *cfg);

/* ------------------------------------------------------------------------ */
/* Group 2c: batching -- many independent grids in one persistent launch     */
/* ------------------------------------------------------------------------ */

typedef struct psb_batch psb_batch;
/* A batch member: a built-in kernel over its own grids for `steps` double-
 * buffered steps (maps in->out then out->in, like PSStencilRun(m1, m2,
 * steps/2)). grids/params as for psb_stencil_map with the full-grid (7-pt)
 * or interior (Himeno) domain. */
psb_status psb_batch_create(psb_batch **b);
psb_status psb_batch_add(psb_batch *b, int kernel_id, __PSGrid *const *grids, int ngrids,
                         const double *params, int nparams, int steps, int *member);
/* Run every member to completion. mode 0: one persistent launch with a
 * device work list; 1: one launch per global step, captured in a CUDA
 * graph; 2: the plain loop, each member alone, one launch per step. */
psb_status psb_batch_run(psb_batch *b, int mode);
psb_status psb_batch_stats(psb_batch *b, double *device_ms, int64_t *launches,
                           int64_t *lattice_updates);
/* Stop a member early once its relative residual is <= tol, checked every
 * check_every steps (7-point: |u_{n+1}-u_n|_2 / |u_{n+1}|_2; Himeno:
 * sqrt(gosa_n / gosa_0)); modes 0 and 1 only. */
psb_status psb_batch_set_stop(psb_batch *b, int member, double tol, int check_every);
/* Steps a member completed in the last run, its last residual (as defined
 * above, -1 if never checked) and which of its two grids holds the result
 * (0 or 1). */
psb_status psb_batch_member_result(psb_batch *b, int member, int *steps_done, double *residual,
                                   int *result_grid);
/* How the last mode-0/1 run cut a member into work items (no counterpart in
 * the reference, which has no batching): the points of an item in x and y,
 * its planes in z, the items of one step, and whether consecutive steps of
 * the member overlapped as a wavefront (1: an item waited only for the 27
 * items around it in the previous step; 0: for the whole previous step),
 * whether its bucket has an entry in the autotuner's table (1; the entry
 * may keep the fewest-tiles rule) or not (0: the rule), the sweeps an item
 * advances (t_depth: 2 for
 * Himeno members that run two sweeps per pass) and the member's units of
 * work in the launch (steps, or passes when t_depth is 2). PSB_ERR_INVALID
 * before the batch has run in mode 0 or 1. */
typedef struct {
  int tile_x, tile_y, z_chunk;
  int tiles;
  int wavefront;
  int tuned;
  int t_depth;
  int units;
} psb_batch_layout;
psb_status psb_batch_member_layout(psb_batch *b, int member, psb_batch_layout *layout);
/* Autotune the batch's members (the reference tunes by trial at translation
 * time, translator/reference_translator.cc:749-1223): for each size bucket
 * -- member kind, element type and extents rounded up to powers of two --
 * without a cached entry (every bucket with force != 0), copies of a
 * scratch member of those extents are timed in the persistent kernel over
 * candidate tile widths (Himeno: also two sweeps per pass), the z chunk
 * following the batch's own rule; the fastest is cached in the tune table
 * and its JSON file and used by later mode-0/1 runs for every member of the
 * bucket (the members' own grids are not touched). */
psb_status psb_batch_autotune(psb_batch *b, int force);
/* Batch member shapes live in the tune table (psb_tune_set/psb_tune_get and
 * its JSON cache) under kernel id PSB_BATCH_TUNE_BASE + kernel_id - 1, where
 * kernel_id is the member's stencil (PSB_KERNEL_DIFFUSION7,
 * _DIFFUSION7_PERIODIC or _HIMENO19), type PS_FLOAT, and the member's size
 * bucket (each extent rounded up to a power of two, at least 8). A run
 * uses tile_x (consumer threads along x = tile_x / 4) and, for Himeno,
 * t_depth (2: two sweeps per pass of 64 x 8 tiles); the z chunk follows the
 * batch's own rule. Setting an entry by hand pins the shape of a bucket. */
#define PSB_BATCH_TUNE_BASE 100
psb_status psb_batch_free(psb_batch *b);

/* ------------------------------------------------------------------------ */
/* Group 2d: serving -- continuous batching of solve requests                */
/* ------------------------------------------------------------------------ */

/* A server owns a worker thread that admits queued requests in arrival
 * order while the device-memory budget and the slot limit allow, keeps each
 * admitted request's grids resident on the device until it finishes, and
 * advances all admitted requests together in rounds of the persistent
 * batched kernel (group 2c); requests that arrive while a round runs join at
 * the next round boundary. A request finishes when its relative residual
 * (as for psb_batch_set_stop) is <= tol at a check, or after max_steps.
 * Results do not depend on what else is being served: each request's
 * arithmetic and residual sums are those of serving it alone.
 * mode PSB_SERVE_BATCHED: the above. PSB_SERVE_FIFO: the baseline -- one
 * request at a time in arrival order, one plain-kernel launch per step and
 * a separate residual pass at each check (the reference's loop shape). */
typedef struct psb_server psb_server;
enum { PSB_SERVE_BATCHED = 0, PSB_SERVE_FIFO = 1 };
typedef struct {
  int kernel_id;          /* PSB_KERNEL_DIFFUSION7(_PERIODIC) or PSB_KERNEL_HIMENO19 */
  PSIndex dims[3];
  int max_steps;          /* stop after this many steps (>= 1) */
  double tol;             /* stop when the relative residual is <= tol (0: never) */
  int check_every;        /* residual check interval in steps (>= 1 when tol > 0) */
  const float *init;      /* host initial field (nx*ny*nz floats: u, or Himeno p),
                             or NULL to generate it on the device from seed */
  const float *coef;      /* Himeno: 12*nx*ny*nz floats, the fields a0 a1 a2 a3
                             b0 b1 b2 c0 c1 c2 bnd wrk1 one after another, or NULL
                             to generate them from seed; unused for diffusion */
  float *out;             /* host buffer for the final field (nx*ny*nz), or NULL */
  uint64_t seed;          /* seed of the generated fields */
  double params[PSB_MAX_PARAMS];  /* kernel parameters as for psb_stencil_map */
  int nparams;
} psb_request;
/* Fields generated from seed s (psb_grid_fill kinds): diffusion u uniform in
 * [0,1) with seed s; Himeno p = (z/(nz-1))^2, a0..a2, c0..c2 uniform in
 * [0.9,1.1), a3 in [0.95/6,1.05/6), b0..b2 in [-0.01,0.01) with seeds
 * s*16+1 .. s*16+10 in field order, bnd 1 inside and 0 on the faces, wrk1 0. */
typedef struct {
  int64_t id;
  psb_status status;      /* PSB_OK, PSB_ERR_CANCELLED or the failure */
  int steps_done;
  double residual;        /* last relative residual, -1 if never checked */
  double submit_s, start_s, finish_s;  /* host steady clock, seconds */
  int wave_rounds;        /* rounds in which its steps overlapped as a wavefront
                             (psb_batch_layout.wavefront) */
} psb_result;
/* max_slots: requests advanced at once (0: no limit). The budget covers
 * every resident grid, including those of finished requests whose results
 * are still being copied out. */
psb_status psb_server_create(size_t mem_budget_bytes, int max_slots, int mode,
                             psb_server **s);
/* Queue a request. init, coef and out must stay valid until the request
 * completes (psb_server_wait returned it). A request whose grids alone
 * exceed the budget is refused with PSB_ERR_NOMEM. */
psb_status psb_server_submit(psb_server *s, const psb_request *req, int64_t *id);
/* Cancel a queued or running request; it completes with PSB_ERR_CANCELLED
 * (a running one at its next round boundary). */
psb_status psb_server_cancel(psb_server *s, int64_t id);
/* Wait for request id (id < 0: the earliest completed one not yet returned)
 * and return its record; each request is returned once. timeout_s < 0 waits
 * forever; PSB_ERR_TIMEOUT if it did not complete in time. */
psb_status psb_server_wait(psb_server *s, int64_t id, double timeout_s, psb_result *res);
/* Bytes a request needs on the device (its resident grids). */
psb_status psb_server_request_bytes(const psb_request *req, size_t *bytes);
psb_status psb_server_stats(psb_server *s, int64_t *completed, int64_t *rounds,
                            int64_t *launches, size_t *peak_bytes, double *device_ms);
/* Finish every queued and running request, then stop the worker. */
psb_status psb_server_destroy(psb_server *s);

#ifdef __cplusplus
}
#endif

#endif /* PHYSIS_B200_H_ */
