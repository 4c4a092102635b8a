// Runtime core: initialisation, error state, grid allocation and copies.
//
// Drop-in counterparts of runtime/libphysis_rt_cuda.cc (PSInit, __PSGridNew,
// __PSGridFree, __PSGridCopyin/out, __PSGridSet, PSDomain*New,
// __PSCheckCudaError) and runtime/runtime_common.cc (__ps_trace,
// __PSRandomInit). Differences from the reference, by design:
//  - one non-blocking runtime stream instead of the legacy default stream;
//  - translator-free constructors (PSGrid3DFloatNew ...) allocate pitched
//    grids with 128-byte rows and a resident halo;
//  - group-2 (psb_*) calls return a status instead of exiting.
#include <stdarg.h>
#include <string.h>
#include <sys/time.h>
#include <time.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "internal.h"

FILE *__ps_trace = nullptr;

namespace psb {

static Runtime g_rt;
Runtime &rt() { return g_rt; }

double now_s() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}

psb_status set_status(psb_status s) {
  rt().last_status = s;
  return s;
}

psb_status cuda_status(cudaError_t e, const char *what) {
  if (__ps_trace) fprintf(__ps_trace, "physis_b200: %s: %s\n", what, cudaGetErrorString(e));
  // Clear a non-sticky error so it is not reported again by a later call.
  cudaGetLastError();
  snprintf(rt().last_error, sizeof(rt().last_error), "%s: %s", what, cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return set_status(PSB_ERR_NOMEM);
  return set_status(PSB_ERR_CUDA);
}

void fatal_cuda(cudaError_t e, const char *file, int line) {
  // Same behaviour as CUDA_SAFE_CALL in runtime/runtime_common_cuda.h:16-23.
  fprintf(stderr, "CUDA ERROR at %s#%d: %s\n", file, line, cudaGetErrorString(e));
  exit(EXIT_FAILURE);
}

int type_size(int type) {
  switch (type) {
    case PS_INT: return 4;
    case PS_LONG: return 8;
    case PS_FLOAT: return 4;
    case PS_DOUBLE: return 8;
    default: return 0;
  }
}

int type_from_size(int elm_size) {
  if (elm_size == 4) return PS_FLOAT;
  if (elm_size == 8) return PS_DOUBLE;
  return -1;
}

psb_status ensure_init() {
  Runtime &r = rt();
  if (r.inited) return PSB_OK;
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  if (r.inited) return PSB_OK;
  const char *dev = getenv("PHYSIS_B200_DEVICE");
  r.device = dev ? atoi(dev) : 0;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev <= r.device) {
    fprintf(stderr, "physis_b200: no CUDA device %d (%s)\n", r.device,
            e == cudaSuccess ? "not present" : cudaGetErrorString(e));
    return set_status(PSB_ERR_CUDA);
  }
  PSB_TRY(cudaSetDevice(r.device));
  cudaDeviceProp prop;
  PSB_TRY(cudaGetDeviceProperties(&prop, r.device));
  // The kernels are built for sm_100a only; refuse anything else up front
  // (the reference checks for >= 2.0 in runtime_common_cuda.h:61-80).
  if (prop.major != 10) {
    fprintf(stderr, "physis_b200: device %d is sm_%d%d; this build needs sm_100\n", r.device,
            prop.major, prop.minor);
    return set_status(PSB_ERR_UNSUPPORTED);
  }
  r.sm_count = prop.multiProcessorCount;
  r.smem_optin = prop.sharedMemPerBlockOptin;
  PSB_TRY(cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking));
  PSB_TRY(cudaEventCreate(&r.ev_start));
  PSB_TRY(cudaEventCreate(&r.ev_stop));
  PSB_TRY(cudaEventCreateWithFlags(&r.ev_join, cudaEventDisableTiming));
  PSB_TRY(cudaMalloc(&r.d_error, sizeof(int) * 4));
  PSB_TRY(cudaMemset(r.d_error, 0, sizeof(int) * 4));
  const char *impl = getenv("PHYSIS_B200_IMPL");
  if (impl) {
    if (!strcmp(impl, "plain")) r.impl = PSB_IMPL_PLAIN;
    else if (!strcmp(impl, "tma")) r.impl = PSB_IMPL_TMA;
    else if (!strcmp(impl, "generic")) r.impl = PSB_IMPL_GENERIC;
  }
  const char *fp = getenv("PHYSIS_B200_FP_MODE");
  if (fp && !strcmp(fp, "fma")) r.fp_mode = PSB_FP_FMA;
  const char *graph = getenv("PHYSIS_B200_GRAPH");
  if (graph) r.use_graph = atoi(graph) != 0;
  r.inited = true;
  return PSB_OK;
}

// Generated code launches its kernels on the legacy default stream while the
// runtime works on its own non-blocking stream; these joins give the two the
// ordering the reference has with a single stream.
void legacy_join_in() {
  Runtime &r = rt();
  if (cudaEventRecord(r.ev_join, cudaStreamLegacy) == cudaSuccess)
    cudaStreamWaitEvent(r.stream, r.ev_join, 0);
}

void legacy_join_out() {
  Runtime &r = rt();
  if (cudaEventRecord(r.ev_join, r.stream) == cudaSuccess)
    cudaStreamWaitEvent(cudaStreamLegacy, r.ev_join, 0);
}

// ---------------------------------------------------------------------------
// Grids
// ---------------------------------------------------------------------------

GridView GridImpl::view() const {
  GridView v;
  v.origin = (char *)alloc + origin_off * pub.elm_size;
  v.sy = sy;
  v.sz = sz;
  for (int i = 0; i < 3; i++) v.n[i] = i < pub.num_dims ? pub.dim[i] : 1;
  v.type = type;
  v.halo = layout == PSB_LAYOUT_PITCHED ? halo : 0;
  return v;
}

GridImpl *as_impl(const void *g) {
  if (!g) return nullptr;
  GridImpl *gi = (GridImpl *)g;
  if (gi->magic != 0x50534232u) return nullptr;
  return gi;
}

static void set_dev_struct(GridImpl *g, void *p0) {
  switch (g->pub.num_dims) {
    case 1:
      g->dev.d1.dim[0] = g->pub.dim[0];
      g->dev.d1.p0 = p0;
      break;
    case 2:
      g->dev.d2.dim[0] = g->pub.dim[0];
      g->dev.d2.dim[1] = g->pub.dim[1];
      g->dev.d2.p0 = p0;
      break;
    default:
      g->dev.d3.dim[0] = g->pub.dim[0];
      g->dev.d3.dim[1] = g->pub.dim[1];
      g->dev.d3.dim[2] = g->pub.dim[2];
      g->dev.d3.p0 = p0;
      break;
  }
  g->pub.dev = (__PSGrid_dev *)&g->dev;
}

// Describe a grid (layout and strides; no allocation). Dense: exactly the
// reference layout. Pitched: x rows are padded to 128 bytes with one
// 128-byte line (at least PSB_HALO cells) left of logical x = 0, and
// PSB_HALO halo rows/planes around y and z.
static GridImpl *grid_describe(int type, int elm_size, int nd, const int *dims, int layout) {
  GridImpl *g = new GridImpl();
  g->pub.elm_size = elm_size;
  g->pub.num_dims = nd;
  g->pub.num_elms = 1;
  for (int i = 0; i < PS_MAX_DIM; i++) g->pub.dim[i] = i < nd ? dims[i] : 0;
  for (int i = 0; i < nd; i++) g->pub.num_elms *= dims[i];
  g->type = type;
  int n[3] = {dims[0], nd > 1 ? dims[1] : 1, nd > 2 ? dims[2] : 1};
  if (layout == PSB_LAYOUT_PITCHED && (elm_size == 4 || elm_size == 8)) {
    int line = 128 / elm_size;
    int h = PSB_HALO;
    g->layout = PSB_LAYOUT_PITCHED;
    g->halo = h;
    g->pad_left = line;
    g->pitch = ((int64_t)line + n[0] + h + line - 1) / line * line;
    g->rows = nd > 1 ? n[1] + 2 * h : 1;
    g->planes = nd > 2 ? n[2] + 2 * h : 1;
    g->sy = g->pitch;
    g->sz = g->pitch * g->rows;
    g->origin_off = g->pad_left + (nd > 1 ? h * g->sy : 0) + (nd > 2 ? h * g->sz : 0);
  } else {
    g->layout = PSB_LAYOUT_DENSE;
    g->pitch = n[0];
    g->rows = n[1];
    g->planes = n[2];
    g->sy = n[0];
    g->sz = (int64_t)n[0] * n[1];
    g->origin_off = 0;
  }
  g->alloc_bytes = (size_t)g->pitch * g->rows * g->planes * elm_size;
  return g;
}

// Point a described grid at its allocation; a zero-filled grid has a
// consistent halo for every boundary mode (the interior is zero too).
static void grid_attach(GridImpl *g) {
  g->ghost_valid = g->layout == PSB_LAYOUT_PITCHED ? PSB_BOUNDARY_PERIODIC : PSB_BOUNDARY_NONE;
  g->pub.p0 = (char *)g->alloc + g->origin_off * g->pub.elm_size;
  set_dev_struct(g, g->pub.p0);
}

static psb_status grid_alloc(int type, int elm_size, int nd, const int *dims, int layout,
                             GridImpl **out) {
  *out = nullptr;
  if (nd < 1 || nd > 3) return set_status(PSB_ERR_INVALID);
  for (int i = 0; i < nd; i++)
    if (dims[i] <= 0) return set_status(PSB_ERR_INVALID);
  if (elm_size <= 0) return set_status(PSB_ERR_INVALID);
  PSB_CHECK(ensure_init());
  GridImpl *g = grid_describe(type, elm_size, nd, dims, layout);
  cudaError_t e = cudaMalloc(&g->alloc, g->alloc_bytes);
  if (e != cudaSuccess) {
    delete g;
    cudaGetLastError();
    return cuda_status(e, "cudaMalloc(grid)");
  }
  e = cudaMemsetAsync(g->alloc, 0, g->alloc_bytes, rt().stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(rt().stream);
  if (e != cudaSuccess) {
    cudaFree(g->alloc);
    delete g;
    return cuda_status(e, "cudaMemset(grid)");
  }
  grid_attach(g);
  *out = g;
  return PSB_OK;
}

size_t grid_pitched_bytes(int elm_size, const int *dims) {
  GridImpl *g = grid_describe(PS_FLOAT, elm_size, 3, dims, PSB_LAYOUT_PITCHED);
  const size_t b = g->alloc_bytes;
  delete g;
  return b;
}

psb_status grid_alloc_pool(int type, const int *dims, cudaMemPool_t pool, cudaStream_t s,
                           GridImpl **out) {
  *out = nullptr;
  for (int i = 0; i < 3; i++)
    if (dims[i] <= 0) return set_status(PSB_ERR_INVALID);
  GridImpl *g = grid_describe(type, type_size(type), 3, dims, PSB_LAYOUT_PITCHED);
  cudaError_t e = cudaMallocFromPoolAsync(&g->alloc, g->alloc_bytes, pool, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->alloc, 0, g->alloc_bytes, s);
  if (e != cudaSuccess) {
    if (g->alloc) cudaFreeAsync(g->alloc, s);
    delete g;
    cudaGetLastError();
    return cuda_status(e, "cudaMallocFromPoolAsync(grid)");
  }
  grid_attach(g);
  *out = g;
  return PSB_OK;
}

void grid_free_pool(GridImpl *g, cudaStream_t s) {
  if (!g) return;
  if (g->alloc) cudaFreeAsync(g->alloc, s);
  g->magic = 0;
  delete g;
}

psb_status grid_copy_in_on(GridImpl *g, const void *src, cudaStream_t s) {
  PSB_CHECK(pitched_transfer(g, (void *)src, true, s));
  g->ghost_valid = PSB_BOUNDARY_NONE;
  return PSB_OK;
}

psb_status grid_copy_out_on(GridImpl *g, void *dst, cudaStream_t s) {
  return pitched_transfer(g, dst, false, s);
}

static void grid_free(GridImpl *g) {
  if (!g) return;
  if (g->component) return;  // freed with its user-type grid
  for (GridImpl *c : g->comps) {
    c->component = false;
    grid_free(c);
  }
  g->comps.clear();
  drop_all_graphs();
  maps_forget_grid(g);
  if (g->user_type) {
    if (g->pub.dev && g->user_free) g->user_free(g->pub.dev);
  } else if (g->alloc) {
    cudaStreamSynchronize(rt().stream);
    PSB_FATAL(cudaFree(g->alloc));
  }
  g->magic = 0;
  delete g;
}

static psb_status copy_in(GridImpl *g, const void *src, bool sync) {
  Runtime &r = rt();
  legacy_join_in();
  int E = g->pub.elm_size;
  if (!g->comps.empty()) {
    PSB_CHECK(user_transfer(g, (void *)src, true, r.stream));
  } else if (g->layout == PSB_LAYOUT_DENSE) {
    PSB_TRY(cudaMemcpyAsync(g->alloc, src, (size_t)g->pub.num_elms * E, cudaMemcpyHostToDevice,
                            r.stream));
  } else {
    PSB_CHECK(pitched_transfer(g, (void *)src, true, r.stream));
    g->ghost_valid = PSB_BOUNDARY_NONE;
  }
  if (sync) PSB_TRY(cudaStreamSynchronize(r.stream));
  return PSB_OK;
}

static psb_status copy_out(GridImpl *g, void *dst, bool sync) {
  Runtime &r = rt();
  legacy_join_in();
  int E = g->pub.elm_size;
  if (!g->comps.empty()) {
    PSB_CHECK(user_transfer(g, dst, false, r.stream));
  } else if (g->layout == PSB_LAYOUT_DENSE) {
    PSB_TRY(cudaMemcpyAsync(dst, g->alloc, (size_t)g->pub.num_elms * E, cudaMemcpyDeviceToHost,
                            r.stream));
  } else {
    PSB_CHECK(pitched_transfer(g, dst, false, r.stream));
  }
  if (sync) PSB_TRY(cudaStreamSynchronize(r.stream));
  return PSB_OK;
}

// Read the device error word written by bounded waits; clears it.
static psb_status check_device_error() {
  int err = 0;
  if (!rt().d_error) return PSB_OK;
  cudaError_t e = cudaMemcpy(&err, rt().d_error, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, "read error word");
  if (err) {
    cudaMemset(rt().d_error, 0, sizeof(int));
    return set_status(PSB_ERR_TIMEOUT);
  }
  // Word 1: a compiled stencil's read outside its grid.
  e = cudaMemcpy(&err, rt().d_error + 1, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, "read error word");
  if (err) {
    cudaMemset(rt().d_error + 1, 0, sizeof(int));
    return set_status(PSB_ERR_BOUNDS);
  }
  return PSB_OK;
}

// ---------------------------------------------------------------------------
// TMA descriptors
// ---------------------------------------------------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

bool tma_eligible(const GridImpl *g) {
  if (g->user_type || !g->comps.empty() || g->pub.num_dims != 3) return false;
  if (g->pub.elm_size != 4 && g->pub.elm_size != 8) return false;
  if (((uintptr_t)g->alloc & 15) != 0) return false;
  if ((g->sy * g->pub.elm_size) % 16 != 0) return false;
  if ((g->sz * g->pub.elm_size) % 16 != 0) return false;
  return true;
}

psb_status get_tmap(GridImpl *g, int bx, int by, const CUtensorMap **out, int l2_promotion) {
  uint64_t key = ((uint64_t)l2_promotion << 48) | ((uint64_t)bx << 24) | (uint32_t)by;
  auto it = g->tmaps.find(key);
  if (it != g->tmaps.end()) {
    *out = &it->second;
    return PSB_OK;
  }
  EncodeTiledFn fn = encode_fn();
  if (!fn || !tma_eligible(g)) return set_status(PSB_ERR_UNSUPPORTED);
  CUtensorMap m;
  int E = g->pub.elm_size;
  CUtensorMapDataType dt = E == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  // The x extent ends at the right halo, not at the padded pitch: box columns
  // past it are out of bounds, so TMA fills them instead of reading padding
  // from DRAM (this matters for narrow grids, whose rows are mostly padding).
  const int64_t xext = g->layout == PSB_LAYOUT_PITCHED
                           ? std::min<int64_t>(g->pitch, (int64_t)g->pad_left + g->pub.dim[0] + g->halo)
                           : g->pitch;
  cuuint64_t dims[3] = {(cuuint64_t)xext, (cuuint64_t)g->rows, (cuuint64_t)g->planes};
  cuuint64_t strides[2] = {(cuuint64_t)(g->sy * E), (cuuint64_t)(g->sz * E)};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  // The whole allocation is described; kernels address it in allocation
  // coordinates (logical + (pad_left, halo, halo)).
  CUresult res = fn(&m, dt, 3, g->alloc, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, (CUtensorMapL2promotion)l2_promotion,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (res != CUDA_SUCCESS) return set_status(PSB_ERR_UNSUPPORTED);
  auto ins = g->tmaps.emplace(key, m);
  *out = &ins.first->second;
  return PSB_OK;
}

}  // namespace psb

using namespace psb;

// ===========================================================================
// C ABI, group 1
// ===========================================================================
extern "C" {

void PSInit(int *argc, char ***argv, int grid_num_dims, ...) {
  (void)grid_num_dims;
  // --physis-trace (runtime/runtime.cc:81-91): strip it and trace to stderr.
  __ps_trace = nullptr;
  if (argc && argv && *argv) {
    int w = 0;
    for (int i = 0; i < *argc; i++) {
      const char *a = (*argv)[i];
      if (a && (!strcmp(a, "-physis-trace") || !strcmp(a, "--physis-trace"))) {
        __ps_trace = stderr;
        continue;
      }
      (*argv)[w++] = (*argv)[i];
    }
    *argc = w;
  }
  if (getenv("PHYSIS_B200_TRACE")) __ps_trace = stderr;
  psb_status s = ensure_init();
  if (s != PSB_OK) {
    fprintf(stderr, "physis_b200: initialisation failed: %s\n", psb_status_string(s));
    exit(EXIT_FAILURE);
  }
  if (__ps_trace) fprintf(__ps_trace, "Physis: Tracing enabled\n");
}

void PSFinalize(void) {
  Runtime &r = rt();
  if (!r.inited) return;
  cudaStreamSynchronize(r.stream);
  for (auto &kv : r.graphs) cudaGraphExecDestroy(kv.second);
  r.graphs.clear();
  for (auto &m : r.maps) {
    if (m.d_partials) cudaFree(m.d_partials);
    if (m.d_ticket) cudaFree(m.d_ticket);
    // d_counter points into the d_ticket allocation.
    if (m.d_history) cudaFree(m.d_history);
  }
  r.maps.clear();
  for (auto &d : r.generics)
    if (d.dev) cudaFree(d.dev);
  r.generics.clear();
  cudaEventDestroy(r.ev_start);
  cudaEventDestroy(r.ev_stop);
  cudaEventDestroy(r.ev_join);
  cudaFree(r.d_error);
  cudaStreamDestroy(r.stream);
  r.d_error = nullptr;
  r.stream = nullptr;
  r.inited = false;
}

int __PSGridGetID(__PSGrid *g) {
  (void)g;
  return 0;
}

__PSGrid *__PSGridNew(int elm_size, int num_dims, PSVectorInt dim, __PSGrid_devNewFunc func) {
  if (ensure_init() != PSB_OK) {
    fprintf(stderr, "physis_b200: runtime not initialised\n");
    exit(EXIT_FAILURE);
  }
  if (func) {
    // User-defined point type: the generated allocator owns the device
    // memory (libphysis_rt_cuda.cc:63-65).
    GridImpl *g = new GridImpl();
    g->pub.elm_size = elm_size;
    g->pub.num_dims = num_dims;
    g->pub.num_elms = 1;
    for (int i = 0; i < PS_MAX_DIM; i++) g->pub.dim[i] = i < num_dims ? dim[i] : 0;
    for (int i = 0; i < num_dims; i++) g->pub.num_elms *= dim[i];
    g->user_type = true;
    g->pub.dev = (__PSGrid_dev *)func(num_dims, dim);
    g->pub.p0 = nullptr;
    return &g->pub;
  }
  GridImpl *g = nullptr;
  psb_status s = grid_alloc(type_from_size(elm_size), elm_size, num_dims, dim, PSB_LAYOUT_DENSE, &g);
  if (s == PSB_ERR_NOMEM || s == PSB_ERR_INVALID) return INVALID_GRID;
  if (s != PSB_OK) {
    fprintf(stderr, "physis_b200: grid allocation failed: %s\n", psb_status_string(s));
    exit(EXIT_FAILURE);
  }
  return &g->pub;
}

void __PSGridFree(__PSGrid *p, __PSGrid_devFreeFunc func) {
  GridImpl *g = as_impl(p);
  if (!g) return;
  if (g->user_type) g->user_free = func;
  grid_free(g);
}

void __PSGridCopyin(void *p, const void *src_array, __PSGrid_devCopyinFunc func) {
  GridImpl *g = as_impl(p);
  if (!g) return;
  if (func) {
    func(g->pub.dev, src_array);
    return;
  }
  psb_status s = copy_in(g, src_array, true);
  if (s != PSB_OK) {
    fprintf(stderr, "CUDA ERROR: grid copy-in failed: %s\n", psb_status_string(s));
    exit(EXIT_FAILURE);
  }
}

void __PSGridCopyout(void *p, void *dst_array, __PSGrid_devCopyoutFunc func) {
  GridImpl *g = as_impl(p);
  if (!g) return;
  if (func) {
    func(g->pub.dev, dst_array);
    return;
  }
  psb_status s = copy_out(g, dst_array, true);
  if (s == PSB_OK) s = check_device_error();
  if (s != PSB_OK) {
    fprintf(stderr, "CUDA ERROR: grid copy-out failed: %s\n", psb_status_string(s));
    exit(EXIT_FAILURE);
  }
}

void __PSGridSwap(__PSGrid *g) { (void)g; }
void __PSGridMirror(__PSGrid *g) { (void)g; }

PSDomain1D PSDomain1DNew(PSIndex minx, PSIndex maxx) {
  PSDomain1D d;
  memset(&d, 0, sizeof(d));
  d.min[0] = d.local_min[0] = minx;
  d.max[0] = d.local_max[0] = maxx;
  return d;
}

PSDomain2D PSDomain2DNew(PSIndex minx, PSIndex maxx, PSIndex miny, PSIndex maxy) {
  PSDomain2D d;
  memset(&d, 0, sizeof(d));
  d.min[0] = d.local_min[0] = minx;
  d.max[0] = d.local_max[0] = maxx;
  d.min[1] = d.local_min[1] = miny;
  d.max[1] = d.local_max[1] = maxy;
  return d;
}

PSDomain3D PSDomain3DNew(PSIndex minx, PSIndex maxx, PSIndex miny, PSIndex maxy, PSIndex minz,
                         PSIndex maxz) {
  PSDomain3D d;
  d.min[0] = d.local_min[0] = minx;
  d.max[0] = d.local_max[0] = maxx;
  d.min[1] = d.local_min[1] = miny;
  d.max[1] = d.local_max[1] = maxy;
  d.min[2] = d.local_min[2] = minz;
  d.max[2] = d.local_max[2] = maxz;
  return d;
}

static int64_t element_offset(GridImpl *g, va_list vl, bool *ok) {
  int64_t idx[3] = {0, 0, 0};
  *ok = true;
  for (int i = 0; i < g->pub.num_dims; i++) {
    PSIndex v = va_arg(vl, PSIndex);
    if (v < 0 || v >= g->pub.dim[i]) *ok = false;
    idx[i] = v;
  }
  return g->origin_off + idx[0] + idx[1] * g->sy + idx[2] * g->sz;
}

void __PSGridSet(__PSGrid *p, void *buf, ...) {
  GridImpl *g = as_impl(p);
  if (!g || g->user_type || !g->comps.empty()) return;
  va_list vl;
  va_start(vl, buf);
  bool ok;
  int64_t off = element_offset(g, vl, &ok);
  va_end(vl);
  if (!ok) {
    fprintf(stderr, "physis_b200: __PSGridSet index out of range\n");
    exit(EXIT_FAILURE);
  }
  legacy_join_in();
  PSB_FATAL(cudaMemcpyAsync((char *)g->alloc + off * g->pub.elm_size, buf, g->pub.elm_size,
                            cudaMemcpyHostToDevice, rt().stream));
  PSB_FATAL(cudaStreamSynchronize(rt().stream));
  if (g->layout == PSB_LAYOUT_PITCHED) g->ghost_valid = PSB_BOUNDARY_NONE;
}

void __PSGridGet(__PSGrid *p, void *buf, ...) {
  GridImpl *g = as_impl(p);
  if (!g || g->user_type || !g->comps.empty()) return;
  va_list vl;
  va_start(vl, buf);
  bool ok;
  int64_t off = element_offset(g, vl, &ok);
  va_end(vl);
  if (!ok) {
    fprintf(stderr, "physis_b200: __PSGridGet index out of range\n");
    exit(EXIT_FAILURE);
  }
  legacy_join_in();
  PSB_FATAL(cudaMemcpyAsync(buf, (char *)g->alloc + off * g->pub.elm_size, g->pub.elm_size,
                            cudaMemcpyDeviceToHost, rt().stream));
  PSB_FATAL(cudaStreamSynchronize(rt().stream));
}

void __PSCheckCudaError(const char *message) {
  cudaError_t error = cudaGetLastError();
  if (error != cudaSuccess) {
    fprintf(stderr, "ERROR: %s: %s\n", message, cudaGetErrorString(error));
    exit(1);
  }
}

void *__PSRandomInit(int n) {
  // A random permutation of 0..n-1 (runtime_common.cc:35-50), drawn with a
  // seeded xorshift so that it does not disturb the process's rand state.
  int *h = (int *)calloc(n > 0 ? n : 1, sizeof(int));
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  uint64_t s = (uint64_t)tv.tv_usec * 2654435761u + 1;
  for (int i = 0; i < n; i++) h[i] = i;
  for (int i = n - 1; i > 0; i--) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    int j = (int)(s % (uint64_t)(i + 1));
    int t = h[i];
    h[i] = h[j];
    h[j] = t;
  }
  return h;
}

// ===========================================================================
// Group 2a: translator-free constructors and copies
// ===========================================================================

static __PSGrid *new_pitched(int type, int nd, int nx, int ny, int nz) {
  int dims[3] = {nx, ny, nz};
  GridImpl *g = nullptr;
  psb_status s = grid_alloc(type, type_size(type), nd, dims, PSB_LAYOUT_PITCHED, &g);
  if (s != PSB_OK) return INVALID_GRID;
  return &g->pub;
}

#define PSB_DEFINE_NEW(NAME, TYPE)                                                       \
  __PSGrid *PSGrid1D##NAME##New(PSIndex nx, ...) { return new_pitched(TYPE, 1, nx, 1, 1); } \
  __PSGrid *PSGrid2D##NAME##New(PSIndex nx, PSIndex ny, ...) {                          \
    return new_pitched(TYPE, 2, nx, ny, 1);                                              \
  }                                                                                      \
  __PSGrid *PSGrid3D##NAME##New(PSIndex nx, PSIndex ny, PSIndex nz, ...) {              \
    return new_pitched(TYPE, 3, nx, ny, nz);                                             \
  }
PSB_DEFINE_NEW(Float, PS_FLOAT)
PSB_DEFINE_NEW(Double, PS_DOUBLE)
PSB_DEFINE_NEW(Int, PS_INT)
PSB_DEFINE_NEW(Long, PS_LONG)

void PSGridCopyin(void *g, const void *src_array) { __PSGridCopyin(g, src_array, nullptr); }
void PSGridCopyout(void *g, void *dst_array) { __PSGridCopyout(g, dst_array, nullptr); }
void PSGridFree(void *g) { __PSGridFree((__PSGrid *)g, nullptr); }

// ===========================================================================
// Group 2b: status API
// ===========================================================================

psb_status psb_init(void) { return ensure_init(); }
psb_status PSGetLastError(void) { return rt().last_status; }

const char *psb_status_string(psb_status s) {
  switch (s) {
    case PSB_OK: return "ok";
    case PSB_ERR_INVALID: return "invalid argument";
    case PSB_ERR_NOMEM: return "out of device memory or budget";
    case PSB_ERR_CUDA: return "CUDA error";
    case PSB_ERR_NOT_INIT: return "runtime not initialised";
    case PSB_ERR_TIMEOUT: return "device-side wait timed out";
    case PSB_ERR_UNSUPPORTED: return "unsupported";
    case PSB_ERR_CANCELLED: return "cancelled";
    case PSB_ERR_BUSY: return "busy";
    case PSB_ERR_BOUNDS: return "read outside the grid";
  }
  return "unknown";
}

psb_status psb_grid_new_user(int num_dims, const PSIndex *dims, const psb_user_type *ut,
                             __PSGrid **out) {
  if (!out || !dims || !ut || num_dims < 1 || num_dims > 3) return set_status(PSB_ERR_INVALID);
  *out = nullptr;
  if (ut->nfields < 1 || ut->nfields > PSB_MAX_FIELDS || ut->record_bytes == 0)
    return set_status(PSB_ERR_INVALID);
  int ncomp = 0;
  for (int f = 0; f < ut->nfields; f++) {
    const int es = type_size(ut->field_type[f]);
    if (es == 0 || ut->field_count[f] < 1 || ut->field_offset[f] % es != 0 ||
        ut->field_offset[f] + (size_t)es * ut->field_count[f] > ut->record_bytes)
      return set_status(PSB_ERR_INVALID);
    ncomp += ut->field_count[f];
  }
  if (ncomp > PSB_MAX_COMPONENTS) return set_status(PSB_ERR_INVALID);
  int d[3] = {1, 1, 1};
  for (int i = 0; i < num_dims; i++) {
    if (dims[i] <= 0) return set_status(PSB_ERR_INVALID);
    d[i] = dims[i];
  }
  PSB_CHECK(ensure_init());
  GridImpl *g = new GridImpl();
  g->pub.elm_size = (int)ut->record_bytes;
  g->pub.num_dims = num_dims;
  g->pub.num_elms = 1;
  for (int i = 0; i < PS_MAX_DIM; i++) g->pub.dim[i] = i < num_dims ? d[i] : 0;
  for (int i = 0; i < num_dims; i++) g->pub.num_elms *= d[i];
  g->type = PS_USER;
  g->layout = PSB_LAYOUT_PITCHED;
  g->utype = *ut;
  for (int f = 0; f < ut->nfields; f++) {
    g->comp_field_first.push_back((int)g->comps.size());
    for (int k = 0; k < ut->field_count[f]; k++) {
      GridImpl *c = nullptr;
      psb_status s = grid_alloc(ut->field_type[f], type_size(ut->field_type[f]), num_dims, d,
                                PSB_LAYOUT_PITCHED, &c);
      if (s != PSB_OK) {
        grid_free(g);
        return set_status(s);
      }
      c->component = true;
      g->comps.push_back(c);
    }
  }
  *out = &g->pub;
  return PSB_OK;
}

psb_status psb_grid_component(__PSGrid *p, int field, int index, __PSGrid **out) {
  GridImpl *g = as_impl(p);
  if (!g || !out || g->comps.empty() || field < 0 || field >= g->utype.nfields || index < 0 ||
      index >= g->utype.field_count[field])
    return set_status(PSB_ERR_INVALID);
  *out = &g->comps[g->comp_field_first[field] + index]->pub;
  return PSB_OK;
}

psb_status psb_grid_new(int type, int num_dims, const PSIndex *dims, int layout, __PSGrid **out) {
  if (!out || !dims || type_size(type) == 0) return set_status(PSB_ERR_INVALID);
  int d[3] = {0, 0, 0};
  for (int i = 0; i < num_dims && i < 3; i++) d[i] = dims[i];
  GridImpl *g = nullptr;
  psb_status s = grid_alloc(type, type_size(type), num_dims, d, layout, &g);
  *out = g ? &g->pub : nullptr;
  return s;
}

psb_status psb_grid_layout(const __PSGrid *p, int64_t *stride_y, int64_t *stride_z, int *layout,
                           int64_t *alloc_bytes) {
  GridImpl *g = as_impl(p);
  if (!g) return set_status(PSB_ERR_INVALID);
  if (stride_y) *stride_y = g->sy;
  if (stride_z) *stride_z = g->sz;
  if (layout) *layout = g->layout;
  if (alloc_bytes) *alloc_bytes = (int64_t)g->alloc_bytes;
  return PSB_OK;
}

psb_status psb_grid_copyin_async(__PSGrid *p, const void *src) {
  GridImpl *g = as_impl(p);
  if (!g || g->user_type || !src) return set_status(PSB_ERR_INVALID);
  return copy_in(g, src, false);
}

psb_status psb_grid_copyout_async(__PSGrid *p, void *dst) {
  GridImpl *g = as_impl(p);
  if (!g || g->user_type || !dst) return set_status(PSB_ERR_INVALID);
  return copy_out(g, dst, false);
}

psb_status psb_sync(void) {
  PSB_CHECK(ensure_init());
  PSB_TRY(cudaStreamSynchronize(rt().stream));
  return check_device_error();
}

psb_status psb_host_alloc(size_t bytes, void **ptr) {
  if (!ptr) return set_status(PSB_ERR_INVALID);
  PSB_CHECK(ensure_init());
  PSB_TRY(cudaHostAlloc(ptr, bytes ? bytes : 1, cudaHostAllocPortable));
  return PSB_OK;
}

psb_status psb_host_free(void *ptr) {
  if (ptr) PSB_TRY(cudaFreeHost(ptr));
  return PSB_OK;
}

psb_status psb_grid_copy(__PSGrid *pd, const __PSGrid *ps) {
  GridImpl *d = as_impl(pd), *s = as_impl(ps);
  if (!d || !s || d->pub.elm_size != s->pub.elm_size || d->pub.num_dims != s->pub.num_dims ||
      !d->comps.empty() || !s->comps.empty() || d->user_type || s->user_type)
    return set_status(PSB_ERR_INVALID);
  for (int i = 0; i < d->pub.num_dims; i++)
    if (d->pub.dim[i] != s->pub.dim[i]) return set_status(PSB_ERR_INVALID);
  int E = d->pub.elm_size;
  int nd = d->pub.num_dims;
  cudaMemcpy3DParms p;
  memset(&p, 0, sizeof(p));
  p.srcPtr = make_cudaPitchedPtr(s->alloc, (size_t)s->pitch * E, s->pitch, s->rows);
  p.srcPos = make_cudaPos((size_t)s->pad_left * E, nd > 1 ? s->halo : 0, nd > 2 ? s->halo : 0);
  p.dstPtr = make_cudaPitchedPtr(d->alloc, (size_t)d->pitch * E, d->pitch, d->rows);
  p.dstPos = make_cudaPos((size_t)d->pad_left * E, nd > 1 ? d->halo : 0, nd > 2 ? d->halo : 0);
  p.extent = make_cudaExtent((size_t)d->pub.dim[0] * E, nd > 1 ? d->pub.dim[1] : 1,
                             nd > 2 ? d->pub.dim[2] : 1);
  p.kind = cudaMemcpyDeviceToDevice;
  PSB_TRY(cudaMemcpy3DAsync(&p, rt().stream));
  d->ghost_valid = PSB_BOUNDARY_NONE;
  return PSB_OK;
}

}  // extern "C"
