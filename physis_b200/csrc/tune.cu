// Runtime autotuner for the built-in stencil kernels.
//
// The reference tunes at translation time: physisc emits one shared object
// per optimisation-flag pattern and a dlopen trial loop that times each one
// (translator/reference_translator.cc:749-1223, physisc.cc:600-655). Here the
// tuner runs inside the runtime: for a (kernel, element type, nx, ny, nz)
// key it times every candidate tile shape of the TMA kernel (tile x/y, z
// chunk, ring depth) and the plain kernel on scratch grids of that shape with
// CUDA events, keeps the fastest, and caches the choice in a JSON file
// ($PHYSIS_B200_TUNE_CACHE, default ~/.cache/physis_b200_tune.json) so later
// processes start tuned. PSStencilRun looks configurations up here.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <dlfcn.h>
#include <sys/stat.h>

#include <algorithm>
#include <string>
#include <vector>

#include "internal.h"

namespace psb {

bool TuneKey::operator<(const TuneKey &o) const {
  if (kernel != o.kernel) return kernel < o.kernel;
  if (type != o.type) return type < o.type;
  if (nx != o.nx) return nx < o.nx;
  if (ny != o.ny) return ny < o.ny;
  return nz < o.nz;
}

psb_tune_config default_config(int kernel, int type, const int *n) {
  psb_tune_config c;
  c.impl = PSB_IMPL_TMA;
  c.t_depth = 1;
  if (kernel == PSB_KERNEL_HIMENO19) {
    c.tile_x = 64;
    c.tile_y = 8;
    c.z_chunk = 32;
    c.stages = 6;
  } else {
    c.tile_x = 32;
    c.tile_y = 16;
    c.z_chunk = 16;
    c.stages = 6;
  }
  // Small grids: shorter chunks (down to 2 planes) keep at least four CTAs
  // per SM in flight; a 64^3 step is launch-bound and runs 3x faster in
  // 2-plane chunks than in 16-plane ones (measured).
  const int64_t tiles = (int64_t)((n[0] + c.tile_x - 1) / c.tile_x) * ((n[1] + c.tile_y - 1) / c.tile_y);
  const int64_t want = (int64_t)rt().sm_count * 4;
  while (c.z_chunk > 2 && tiles * ((n[2] + c.z_chunk - 1) / c.z_chunk) < want) c.z_chunk /= 2;
  return c;
}

static std::string cache_path() {
  const char *p = getenv("PHYSIS_B200_TUNE_CACHE");
  if (p && *p) return p;
  const char *h = getenv("HOME");
  return std::string(h ? h : "/tmp") + "/.cache/physis_b200_tune.json";
}

// The tuned configurations measured on B200 ship next to the library
// (physis_b200/tune_b200.json); a user cache entry for the same key wins.
static std::string shipped_path() {
  Dl_info info;
  if (!dladdr((void *)&shipped_path, &info) || !info.dli_fname) return "";
  std::string so = info.dli_fname;  // .../physis_b200/lib/libphysis_rt_b200.so
  size_t a = so.find_last_of('/');
  if (a == std::string::npos) return "";
  std::string libdir = so.substr(0, a);
  size_t b = libdir.find_last_of('/');
  if (b == std::string::npos) return "";
  return libdir.substr(0, b) + "/tune_b200.json";
}

// Entries are objects {"kernel": ..., "ms": ...} with the keys in the order
// save_cache writes them; any layout of the file (one entry per line, or a
// whole list on one line) is read.
static void parse_cache_file(const std::string &path) {
  Runtime &r = rt();
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return;
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
  fclose(f);
  for (size_t pos = text.find("{\"kernel\""); pos != std::string::npos;
       pos = text.find("{\"kernel\"", pos + 1)) {
    TuneKey k;
    psb_tune_config c;
    double ms = 0;
    int got = sscanf(text.c_str() + pos,
                     "{\"kernel\": %d, \"type\": %d, \"n\": [%d, %d, %d], \"impl\": %d, "
                     "\"tile_x\": %d, \"tile_y\": %d, \"z_chunk\": %d, \"stages\": %d, "
                     "\"t_depth\": %d, \"ms\": %lf",
                     &k.kernel, &k.type, &k.nx, &k.ny, &k.nz, &c.impl, &c.tile_x, &c.tile_y,
                     &c.z_chunk, &c.stages, &c.t_depth, &ms);
    if (got >= 11) r.tune[k] = c;
  }
}

static void load_cache() {
  Runtime &r = rt();
  if (r.tune_loaded) return;
  r.tune_loaded = true;
  r.tune_path = cache_path();
  // PHYSIS_B200_TUNE_SHIPPED=0 leaves the shipped table out (only the user
  // cache and the library's own rules apply).
  const char *use_shipped = getenv("PHYSIS_B200_TUNE_SHIPPED");
  std::string shipped = use_shipped && use_shipped[0] == '0' ? "" : shipped_path();
  if (!shipped.empty()) parse_cache_file(shipped);
  parse_cache_file(r.tune_path);
}

static void save_cache() {
  Runtime &r = rt();
  std::string path = r.tune_path.empty() ? cache_path() : r.tune_path;
  std::string dir = path.substr(0, path.find_last_of('/'));
  if (!dir.empty()) {
    std::string cmd = dir;
    // Create the directory one level deep (the usual ~/.cache case).
    mkdir(cmd.c_str(), 0755);
  }
  std::string tmp = path + ".tmp";
  FILE *f = fopen(tmp.c_str(), "w");
  if (!f) return;
  fprintf(f, "[\n");
  size_t i = 0;
  for (auto &kv : r.tune) {
    const TuneKey &k = kv.first;
    const psb_tune_config &c = kv.second;
    fprintf(f,
            "{\"kernel\": %d, \"type\": %d, \"n\": [%d, %d, %d], \"impl\": %d, \"tile_x\": %d, "
            "\"tile_y\": %d, \"z_chunk\": %d, \"stages\": %d, \"t_depth\": %d, \"ms\": 0}%s\n",
            k.kernel, k.type, k.nx, k.ny, k.nz, c.impl, c.tile_x, c.tile_y, c.z_chunk, c.stages,
            c.t_depth, ++i < r.tune.size() ? "," : "");
  }
  fprintf(f, "]\n");
  fclose(f);
  rename(tmp.c_str(), path.c_str());
}

void batch_tune_bucket(const int *n, int *bucket) {
  for (int i = 0; i < 3; i++) {
    int b = 8;
    while (b < n[i] && b < (1 << 30)) b <<= 1;
    bucket[i] = b;
  }
}

bool batch_tune_find(int kind, const int *n, psb_tune_config *cfg) {
  load_cache();
  int b[3];
  batch_tune_bucket(n, b);
  auto it = rt().tune.find(TuneKey{kBatchTuneBase + kind, PS_FLOAT, b[0], b[1], b[2]});
  if (it == rt().tune.end()) return false;
  *cfg = it->second;
  return true;
}

void batch_tune_store(int kind, const int *n, const psb_tune_config &cfg) {
  load_cache();
  int b[3];
  batch_tune_bucket(n, b);
  rt().tune[TuneKey{kBatchTuneBase + kind, PS_FLOAT, b[0], b[1], b[2]}] = cfg;
}

void tune_save() { save_cache(); }

psb_status tune_lookup(int kernel, int type, const int *n, psb_tune_config *cfg) {
  load_cache();
  TuneKey k{kernel, type, n[0], n[1], n[2]};
  auto it = rt().tune.find(k);
  *cfg = it != rt().tune.end() ? it->second : default_config(kernel, type, n);
  return PSB_OK;
}

__global__ void k_fill_pattern(float *p, int64_t n, float scale) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u;
    h ^= h >> 15;
    p[i] = scale * (float)(h & 0xffffff) / 16777216.0f;
  }
}

__global__ void k_fill_pattern_d(double *p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u;
    h ^= h >> 15;
    p[i] = (double)(h & 0xffffff) / 16777216.0;
  }
}

// Time `reps` launches of map m with cfg; returns ms per launch (min of 3
// rounds) or a negative value if the configuration cannot run.
static double time_config(MapImpl &m, const psb_tune_config &cfg, int reps) {
  Runtime &r = rt();
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = -1;
  int64_t launches = 0;
  for (int round = 0; round < 4; round++) {
    cudaEventRecord(a, r.stream);
    for (int i = 0; i < reps; i++) {
      // Two-step (temporally blocked) candidates advance two steps per launch.
      psb_status st;
      if (m.kernel_id == PSB_KERNEL_HIMENO19)
        st = cfg.t_depth == 2 ? himeno_tb2_launch(m, m, m.grids[0], m.grids[1], cfg.z_chunk,
                                                  r.stream, &launches)
                              : himeno_launch(m, cfg, r.stream, &launches);
      else
        st = cfg.t_depth == 2 ? diffusion7_tb2_launch(m, m.grids[0], m.grids[1], cfg.z_chunk,
                                                      r.stream, &launches)
                              : diffusion7_launch(m, cfg, r.stream, &launches);
      if (st != PSB_OK) {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return -1;
      }
    }
    cudaEventRecord(b, r.stream);
    if (cudaEventSynchronize(b) != cudaSuccess) {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      return -1;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    ms /= cfg.t_depth == 2 ? 2 : 1;  // per step
    if (round > 0 && (best < 0 || ms / reps < best)) best = ms / reps;  // round 0 warms up
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (cudaGetLastError() != cudaSuccess) return -1;
  return best;
}

}  // namespace psb

using namespace psb;

extern "C" {

psb_status psb_tune_get(int kernel_id, int type, const PSIndex *dims, psb_tune_config *cfg) {
  if (!dims || !cfg) return set_status(PSB_ERR_INVALID);
  int n[3] = {dims[0], dims[1], dims[2]};
  return tune_lookup(kernel_id, type, n, cfg);
}

psb_status psb_tune_set(int kernel_id, int type, const PSIndex *dims, const psb_tune_config *cfg) {
  if (!dims || !cfg) return set_status(PSB_ERR_INVALID);
  load_cache();
  rt().tune[TuneKey{kernel_id, type, dims[0], dims[1], dims[2]}] = *cfg;
  drop_all_graphs();
  return PSB_OK;
}

psb_status psb_autotune(int kernel_id, int type, const PSIndex *dims, int force,
                        psb_tune_config *cfg) {
  PSB_CHECK(ensure_init());
  if (!dims || !cfg) return set_status(PSB_ERR_INVALID);
  if (kernel_id != PSB_KERNEL_DIFFUSION7 && kernel_id != PSB_KERNEL_DIFFUSION7_PERIODIC &&
      kernel_id != PSB_KERNEL_HIMENO19)
    return set_status(PSB_ERR_UNSUPPORTED);
  if (kernel_id == PSB_KERNEL_HIMENO19 && type != PS_FLOAT) return set_status(PSB_ERR_INVALID);
  if (type != PS_FLOAT && type != PS_DOUBLE) return set_status(PSB_ERR_INVALID);
  load_cache();
  Runtime &r = rt();
  TuneKey key{kernel_id, type, dims[0], dims[1], dims[2]};
  if (!force) {
    auto it = r.tune.find(key);
    if (it != r.tune.end()) {
      *cfg = it->second;
      return PSB_OK;
    }
  }
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  const int ngr = kernel_id == PSB_KERNEL_HIMENO19 ? 14 : 2;
  std::vector<__PSGrid *> gs(ngr, nullptr);
  for (int i = 0; i < ngr; i++) {
    psb_status s = psb_grid_new(type, 3, dims, PSB_LAYOUT_PITCHED, &gs[i]);
    if (s != PSB_OK) {
      for (auto g : gs)
        if (g) PSGridFree(g);
      return set_status(s);
    }
    GridImpl *g = as_impl(gs[i]);
    int64_t n = (int64_t)g->alloc_bytes / g->pub.elm_size;
    if (type == PS_DOUBLE)
      k_fill_pattern_d<<<r.sm_count * 4, 256, 0, r.stream>>>((double *)g->alloc, n);
    else
      k_fill_pattern<<<r.sm_count * 4, 256, 0, r.stream>>>((float *)g->alloc, n,
                                                            i == 5 ? 1.0f / 6.0f : 1.0f);
  }
  MapImpl m;
  m.kernel_id = kernel_id;
  m.ngrids = ngr;
  for (int i = 0; i < ngr; i++) m.grids[i] = as_impl(gs[i]);
  if (kernel_id == PSB_KERNEL_HIMENO19) {
    m.dom = PSDomain3DNew(1, dims[0] - 1, 1, dims[1] - 1, 1, dims[2] - 1);
    m.nparams = 1;
    m.params[0] = 0.8;
  } else {
    m.dom = PSDomain3DNew(0, dims[0], 0, dims[1], 0, dims[2]);
    m.nparams = 7;
    for (int i = 0; i < 6; i++) m.params[i] = 0.1;
    m.params[6] = 0.4;
  }
  if (kernel_id == PSB_KERNEL_DIFFUSION7_PERIODIC) launch_halo_fill(m.grids[0], 1, r.stream);
  cudaStreamSynchronize(r.stream);
  int64_t pts = (int64_t)dims[0] * dims[1] * dims[2];
  int reps = (int)std::max<int64_t>(3, std::min<int64_t>(50, 400000000LL / std::max<int64_t>(pts, 1)));
  std::vector<psb_tune_config> cands;
  psb_tune_config plain = default_config(kernel_id, type, (const int *)dims);
  plain.impl = PSB_IMPL_PLAIN;
  cands.push_back(plain);
  const bool him = kernel_id == PSB_KERNEL_HIMENO19;
  std::vector<int> txs = type == PS_DOUBLE ? std::vector<int>{16, 32, 64}
                                           : std::vector<int>{32, 64, 128};
  std::vector<int> tys = him ? std::vector<int>{4, 8, 16} : std::vector<int>{4, 8, 16, 32};
  std::vector<int> zcs = {2, 4, 8, 16, 32, 64, 128};
  std::vector<int> sts = {4, 6, 8};
  for (int tx : txs)
    for (int ty : tys)
      for (int zc : zcs)
        for (int st : sts) {
          if (zc > dims[2] * 2) continue;
          psb_tune_config c;
          c.impl = PSB_IMPL_TMA;
          c.tile_x = tx;
          c.tile_y = ty;
          c.z_chunk = zc;
          c.stages = st;
          c.t_depth = 1;
          cands.push_back(c);
        }
  // Temporal blocking (two steps per launch; clamped float 7-point only).
  // Its tile fields are a valid single-step configuration too, for maps run
  // alone.
  if (kernel_id == PSB_KERNEL_DIFFUSION7 && type == PS_FLOAT)
    for (int zc : {32, 64, 128}) {
      if (zc > dims[2] * 2) continue;
      psb_tune_config c;
      c.impl = PSB_IMPL_TMA;
      c.tile_x = 128;
      c.tile_y = 8;
      c.z_chunk = zc;
      c.stages = 6;
      c.t_depth = 2;
      cands.push_back(c);
    }
  // Himeno, two sweeps per pass (64 x 8 tiles; the single-sweep fields of
  // the entry are the default shape, used for maps run alone).
  if (kernel_id == PSB_KERNEL_HIMENO19)
    for (int zc : {16, 32, 64}) {
      if (zc > dims[2] * 2) continue;
      psb_tune_config c;
      c.impl = PSB_IMPL_TMA;
      c.tile_x = 64;
      c.tile_y = 8;
      c.z_chunk = zc;
      c.stages = 6;
      c.t_depth = 2;
      cands.push_back(c);
    }
  double best_ms = -1;
  psb_tune_config best = default_config(kernel_id, type, (const int *)dims);
  for (auto &c : cands) {
    double ms = time_config(m, c, reps);
    if (__ps_trace)
      fprintf(__ps_trace, "physis_b200: tune impl=%d tile=%dx%d zc=%d st=%d t=%d: %.4f ms\n",
              c.impl, c.tile_x, c.tile_y, c.z_chunk, c.stages, c.t_depth, ms);
    if (ms > 0 && (best_ms < 0 || ms < best_ms)) {
      best_ms = ms;
      best = c;
    }
  }
  for (auto g : gs) PSGridFree(g);
  psb_status err = psb_sync();
  if (err != PSB_OK) return err;
  r.tune[key] = best;
  save_cache();
  drop_all_graphs();
  *cfg = best;
  return PSB_OK;
}

}  // extern "C"
