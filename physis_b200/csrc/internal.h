// Internal declarations of the B200 runtime (not part of the C ABI).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/physis_b200.h"
#include "views.h"

namespace psb {

// Device-side views (GridView, Dom3) are in views.h.

// ---------------------------------------------------------------------------
// Host-side objects
// ---------------------------------------------------------------------------

struct GridImpl {
  __PSGrid pub;  // must stay first: handles are cast to __PSGrid*
  union {
    __PSGrid1D_dev d1;
    __PSGrid2D_dev d2;
    __PSGrid3D_dev d3;
  } dev;
  int type = -1;
  int layout = PSB_LAYOUT_DENSE;
  void *alloc = nullptr;
  size_t alloc_bytes = 0;
  int64_t sy = 0, sz = 0;     // element strides
  int64_t origin_off = 0;     // elements from alloc to logical (0,0,0)
  int64_t pitch = 0, rows = 0, planes = 0;
  int pad_left = 0;           // x cells left of the origin
  int halo = 0;               // y/z halo cells (and minimum x halo)
  int ghost_valid = PSB_BOUNDARY_NONE;  // which halo content is current
  bool user_type = false;
  __PSGrid_devFreeFunc user_free = nullptr;
  uint32_t magic = 0x50534232u;
  // TMA descriptors built on demand, keyed by box shape.
  std::map<uint64_t, CUtensorMap> tmaps;
  // User-defined point type kept as SoA components (one pitched grid per
  // scalar component, in field order); empty for ordinary grids.
  std::vector<GridImpl *> comps;
  std::vector<int> comp_field_first;  // index of field f's first component
  psb_user_type utype{};
  bool component = false;  // a component of a user-type grid (not freed alone)

  int64_t nelems() const { return pub.num_elms; }
  GridView view() const;
};

GridImpl *as_impl(const void *g);  // nullptr if g is not a grid of ours

struct MapImpl {
  int kernel_id = 0;
  __PSDomain dom;
  GridImpl *grids[PSB_MAX_GRIDS] = {};
  int ngrids = 0;
  double params[PSB_MAX_PARAMS] = {};
  int nparams = 0;
  int color = -1;           // -1 all points; 0 red; 1 black; 2 red then black
  bool live = false;
  // Himeno residual bookkeeping.
  int residual_len = 0;
  double *d_partials = nullptr;  // one per CTA
  unsigned *d_ticket = nullptr;
  unsigned *d_counter = nullptr;
  double *d_history = nullptr;
  int partials_cap = 0;
};

struct GenericDesc {
  psb_generic_stencil host;
  void *dev = nullptr;  // device copy of the compact table
};

// Kernel launch configuration for the fast paths.
struct TuneKey {
  int kernel, type, nx, ny, nz;
  bool operator<(const TuneKey &o) const;
};

struct Runtime {
  bool inited = false;
  int device = 0;
  int sm_count = 148;
  size_t smem_optin = 227 * 1024;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  cudaEvent_t ev_join = nullptr;  // orders the runtime stream with the legacy stream
  int *d_error = nullptr;     // device error word (timeouts)
  psb_status last_status = PSB_OK;
  char last_error[256] = {0};  // text of the last CUDA failure
  int impl = PSB_IMPL_AUTO;
  int fp_mode = PSB_FP_EXACT;
  bool use_graph = true;
  double last_ms = 0.0;
  int64_t last_launches = 0;
  bool last_timed = false;
  std::vector<MapImpl> maps;
  std::vector<GenericDesc> generics;
  std::vector<psb_compiled_stencil> compiled;
  std::map<TuneKey, psb_tune_config> tune;
  bool tune_loaded = false;
  std::string tune_path;
  std::recursive_mutex mu;
  // CUDA graphs of run loops, keyed by the map list and unroll.
  std::map<std::string, cudaGraphExec_t> graphs;
};

Runtime &rt();
// Order the runtime stream after work already queued on the legacy default
// stream (where generated kernels launch), and the reverse.
void legacy_join_in();
void legacy_join_out();
psb_status set_status(psb_status s);
psb_status ensure_init();
psb_status cuda_status(cudaError_t e, const char *what);
// Group-1 style fatal check: print and exit like the reference.
void fatal_cuda(cudaError_t e, const char *file, int line);
#define PSB_FATAL(x)                                   \
  do {                                                 \
    cudaError_t e__ = (x);                             \
    if (e__ != cudaSuccess) ::psb::fatal_cuda(e__, __FILE__, __LINE__); \
  } while (0)
#define PSB_TRY(x)                                                  \
  do {                                                              \
    cudaError_t e__ = (x);                                          \
    if (e__ != cudaSuccess) return ::psb::cuda_status(e__, #x);     \
  } while (0)
#define PSB_CHECK(s)                         \
  do {                                       \
    psb_status s__ = (s);                    \
    if (s__ != PSB_OK) return set_status(s__); \
  } while (0)

int type_size(int type);
int type_from_size(int elm_size);  // float for 4, double for 8

// TMA descriptor of a 3-D (or lower) grid, box (bx, by, 1). Coordinates used
// by kernels are relative to the allocation for pitched grids (origin at
// (pad_left, halo, halo)) and to the logical origin for dense grids.
// l2_promotion: a CUtensorMapL2promotion (how much L2 fetches around each
// box row); boxes whose rows are not 256-byte aligned may want less.
psb_status get_tmap(GridImpl *g, int bx, int by, const CUtensorMap **out,
                    int l2_promotion = CU_TENSOR_MAP_L2_PROMOTION_L2_256B);
bool tma_eligible(const GridImpl *g);

// Stencil launches (one application of map m on the runtime stream).
psb_status launch_map(MapImpl &m, int color, int64_t *launches);
psb_status prepare_ghosts(MapImpl &m);
psb_status launch_halo_fill(GridImpl *g, int mode, cudaStream_t s);

// Pitched 3-D grids in a stream-ordered memory pool (serving): allocation and
// zero fill on stream s, free after the work queued on s.
size_t grid_pitched_bytes(int elm_size, const int *dims);
psb_status grid_alloc_pool(int type, const int *dims, cudaMemPool_t pool, cudaStream_t s,
                           GridImpl **out);
void grid_free_pool(GridImpl *g, cudaStream_t s);
psb_status grid_copy_in_on(GridImpl *g, const void *src, cudaStream_t s);
// Host array of records <-> the SoA components of a user-type grid.
psb_status user_transfer(GridImpl *g, void *host, bool h2d, cudaStream_t s);
// Host <-> pitched grid through a dense staging buffer and a pack kernel.
psb_status pitched_transfer(GridImpl *g, void *host, bool h2d, cudaStream_t s);
// First half of a copy-out: allocate a dense staging buffer and pack the
// grid into it on s (the caller copies it out and frees it with
// cudaFreeAsync, ordered after s).
psb_status pitched_stage_out(GridImpl *g, void **stage, cudaStream_t s);
psb_status grid_copy_out_on(GridImpl *g, void *dst, cudaStream_t s);

// Kernel launchers implemented in the .cu files.
psb_status diffusion7_launch(MapImpl &m, const psb_tune_config &cfg, cudaStream_t s,
                             int64_t *launches);
psb_status himeno_launch(MapImpl &m, const psb_tune_config &cfg, cudaStream_t s,
                         int64_t *launches);
// Two steps of a clamped float 7-point map over a whole pitched grid in one
// launch (temporal blocking): reads in, writes out.
psb_status diffusion7_tb2_launch(MapImpl &m, GridImpl *in, GridImpl *out, int zchunk,
                                 cudaStream_t s, int64_t *launches);
bool himeno_tb2_pair(MapImpl **ms, int n);
psb_status himeno_tb2_launch(MapImpl &m1, MapImpl &m2, GridImpl *in, GridImpl *out,
                             int zchunk, cudaStream_t s, int64_t *launches);
psb_status generic_tma_launch(MapImpl &m, const GenericDesc &gd, int color, cudaStream_t s,
                              int64_t *launches);
void generic_note_impl(int impl);
psb_status generic_launch(MapImpl &m, const GenericDesc &d, int color, cudaStream_t s,
                          int64_t *launches);
psb_status reduce_view(const GridView &v, int type, int op, const Dom3 &dom, double *result,
                       cudaStream_t s);
// Reduce the values generic stencil gd would emit over m's domain (no store).
psb_status generic_reduce(MapImpl &m, const GenericDesc &gd, int op, double *result,
                          cudaStream_t s);

// Drop cached CUDA graphs (they bake grid pointers and tile shapes).
void drop_all_graphs();
void maps_forget_grid(const GridImpl *g);

// Autotuning.
psb_tune_config default_config(int kernel, int type, const int *n);
psb_status tune_lookup(int kernel, int type, const int *n, psb_tune_config *cfg);
// Batched members are tuned per (kernel kind, element type, size bucket):
// each extent rounded up to a power of two. Their entries live in the same
// table and cache file under kernel id kBatchTuneBase + the member kind.
constexpr int kBatchTuneBase = PSB_BATCH_TUNE_BASE;
void batch_tune_bucket(const int *n, int *bucket);
bool batch_tune_find(int kind, const int *n, psb_tune_config *cfg);
void batch_tune_store(int kind, const int *n, const psb_tune_config &cfg);
void tune_save();

// Host monotonic seconds.
double now_s();

// Run-time compilation (rtc.cu): a kernel `name` compiled by NVRTC for
// sm_100a from `source` (which may include the library's device headers),
// cached per device and key; PSB_ERR_UNSUPPORTED when NVRTC, the headers or
// the compile are unavailable (the caller keeps its own kernel).
// The staged form of a compiled stencil (k_generic_tma.cu):
// PSB_ERR_UNSUPPORTED when the map does not fit it (the caller then runs the
// stencil's own launch).
psb_status compiled_staged_launch(MapImpl &m, const psb_compiled_stencil &cd, GridImpl **views,
                                  int color, cudaStream_t s);

bool rtc_available();
psb_status rtc_function(const std::string &key, const std::string &source, const char *name,
                        const std::vector<std::string> &options, int smem_bytes,
                        CUfunction *fn);
psb_status rtc_cached(const std::string &key, CUfunction *fn);  // no compile
psb_status rtc_launch(CUfunction fn, unsigned blocks, unsigned threads, unsigned smem,
                      cudaStream_t s, void **args);

}  // namespace psb
