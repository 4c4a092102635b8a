// Stencil maps, the run loop and reductions.
//
// PSStencilMap binds a kernel, a domain, grids and scalars (the closure the
// translator builds as __PSStencil_<k>, reference_runtime_builder.cc:398-550).
// PSStencilRun runs maps in order `iter` times (the generated
// __PSStencilRun_N, translator/cuda_translator.cc:360-529). Here the loop is
// recorded once into a CUDA graph (unrolled by up to kUnroll iterations) and
// replayed, so small grids are not bound by launch latency; device time is
// measured with CUDA events on the runtime stream.
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <cstdio>
#include <string>

#include "internal.h"

namespace psb {

psb_status generic_upload(GenericDesc &d);

static const int kHandleTag = 0x51000000;
static const int kUnroll = 16;

static MapImpl *map_of(PSStencil h) {
  Runtime &r = rt();
  if ((h & 0xff000000) != kHandleTag) return nullptr;
  int idx = h & 0x00ffffff;
  if (idx < 0 || idx >= (int)r.maps.size() || !r.maps[idx].live) return nullptr;
  return &r.maps[idx];
}

static const GenericDesc *generic_of(int kernel_id) {
  int i = kernel_id - PSB_KERNEL_FIRST_GENERIC;
  if (i < 0 || i >= (int)rt().generics.size()) return nullptr;
  return &rt().generics[i];
}

static const psb_compiled_stencil *compiled_of(int kernel_id) {
  int i = kernel_id - PSB_KERNEL_FIRST_COMPILED;
  if (i < 0 || i >= (int)rt().compiled.size()) return nullptr;
  return &rt().compiled[i];
}

// The grid behind each view of a compiled stencil's map: a primitive grid
// gives one view, a grid of a user-defined point type one per component.
static int compiled_views(const MapImpl &m, const psb_compiled_stencil &d,
                          GridImpl **views) {
  int v = 0;
  for (int i = 0; i < m.ngrids; i++) {
    GridImpl *g = m.grids[i];
    if (d.grid_type[i] == PS_USER) {
      if ((int)g->comps.size() != d.grid_components[i] || v + d.grid_components[i] > PSB_MAX_VIEWS)
        return -1;
      for (GridImpl *c : g->comps) views[v++] = c;
    } else {
      if (v >= PSB_MAX_VIEWS) return -1;
      views[v++] = g;
    }
  }
  return v;
}

// A map of a compiled stencil: grids of the declared types, ranks and
// components, a domain inside every emitted view (reads are bounds-checked
// in the kernel), and no grid that is both emitted and read off the point
// unless red-black ordering separates the two.
static psb_status check_compiled_map(const MapImpl &m, const psb_compiled_stencil &d) {
  if (m.ngrids != d.ngrids || m.nparams != d.nparams) return PSB_ERR_INVALID;
  for (int i = 0; i < d.ngrids; i++) {
    const GridImpl *g = m.grids[i];
    if (d.grid_ndims[i] != g->pub.num_dims) return PSB_ERR_INVALID;
    // Grids of point types (psb_grid_new_user) carry their components.
    if ((d.grid_type[i] == PS_USER) != !g->comps.empty()) return PSB_ERR_INVALID;
  }
  GridImpl *views[PSB_MAX_VIEWS];
  if (compiled_views(m, d, views) != d.nviews) return PSB_ERR_INVALID;
  for (int v = 0; v < d.nviews; v++) {
    const GridImpl *g = views[v];
    if (type_size(d.view_type[v]) != g->pub.elm_size) return PSB_ERR_INVALID;
    if (g->type >= 0 && g->type != d.view_type[v]) return PSB_ERR_INVALID;
  }
  for (int k = 0; k < d.ndims; k++)
    if (m.dom.local_min[k] < 0 || m.dom.local_max[k] < m.dom.local_min[k]) return PSB_ERR_INVALID;
  for (int v = 0; v < d.nviews; v++) {
    if (!d.view_emits[v]) continue;
    const GridImpl *g = views[v];
    for (int k = 0; k < d.ndims; k++)
      if (m.dom.local_max[k] > g->pub.dim[k]) return PSB_ERR_INVALID;
    if (m.color < 0)
      for (int w = 0; w < d.nviews; w++)
        if (views[w] == g && d.view_reads_offset[w]) return PSB_ERR_UNSUPPORTED;
  }
  return PSB_OK;
}

// Expected grid count / types of a kernel.
// writes: false for a kernel-function reduction (nothing is stored, so an
// emitted grid that is also read at offsets is fine).
static psb_status check_map(const MapImpl &m, bool writes = true) {
  switch (m.kernel_id) {
    case PSB_KERNEL_DIFFUSION7:
    case PSB_KERNEL_DIFFUSION7_PERIODIC: {
      if (m.ngrids != 2 || m.nparams != 7) return PSB_ERR_INVALID;
      GridImpl *a = m.grids[0], *b = m.grids[1];
      if (a->pub.num_dims != 3 || b->pub.num_dims != 3) return PSB_ERR_INVALID;
      if (a->pub.elm_size != b->pub.elm_size) return PSB_ERR_INVALID;
      if (a->pub.elm_size != 4 && a->pub.elm_size != 8) return PSB_ERR_INVALID;
      if (a->type == PS_INT || a->type == PS_LONG) return PSB_ERR_INVALID;
      for (int i = 0; i < 3; i++)
        if (a->pub.dim[i] != b->pub.dim[i]) return PSB_ERR_INVALID;
      if (a == b) return PSB_ERR_UNSUPPORTED;  // in-place needs two grids
      for (int i = 0; i < 3; i++)
        if (m.dom.local_min[i] < 0 || m.dom.local_max[i] > a->pub.dim[i]) return PSB_ERR_INVALID;
      return PSB_OK;
    }
    case PSB_KERNEL_HIMENO19: {
      if (m.ngrids != 14 || m.nparams != 1) return PSB_ERR_INVALID;
      for (int i = 0; i < 14; i++) {
        GridImpl *g = m.grids[i];
        if (g->pub.num_dims != 3 || g->pub.elm_size != 4 || g->type == PS_INT) return PSB_ERR_INVALID;
        for (int k = 0; k < 3; k++)
          if (g->pub.dim[k] != m.grids[0]->pub.dim[k]) return PSB_ERR_INVALID;
      }
      if (m.grids[0] == m.grids[1]) return PSB_ERR_UNSUPPORTED;
      for (int i = 0; i < 3; i++)
        if (m.dom.local_min[i] < 1 || m.dom.local_max[i] > m.grids[0]->pub.dim[i] - 1)
          return PSB_ERR_INVALID;
      return PSB_OK;
    }
    default: {
      if (const psb_compiled_stencil *cd = compiled_of(m.kernel_id))
        return check_compiled_map(m, *cd);
      const GenericDesc *gd = generic_of(m.kernel_id);
      if (!gd) return PSB_ERR_INVALID;
      const psb_generic_stencil &d = gd->host;
      if (m.ngrids != d.ngrids) return PSB_ERR_INVALID;
      for (int i = 0; i < d.ngrids; i++) {
        GridImpl *g = m.grids[i];
        if (type_size(d.grid_type[i]) != g->pub.elm_size) return PSB_ERR_INVALID;
        int nd = 0;
        for (int k = 0; k < 3; k++)
          if (d.grid_axes[i][k] >= 0) nd = k + 1;
        if (nd != g->pub.num_dims) return PSB_ERR_INVALID;
      }
      // Plain (unwrapped) reads must stay inside the grid for every point of
      // the domain; the reference leaves this undefined, here it is refused.
      {
        auto in_bounds = [&](const psb_factor &f) {
          if (f.grid < 0 || f.boundary != PSB_BOUNDARY_NONE) return true;
          const GridImpl *g = m.grids[f.grid];
          for (int k = 0; k < 3; k++) {
            int ax = d.grid_axes[f.grid][k];
            if (ax < 0) break;
            int lo = m.dom.local_min[ax] + f.offset[ax];
            int hi = m.dom.local_max[ax] - 1 + f.offset[ax];
            if (m.dom.local_max[ax] > m.dom.local_min[ax] && (lo < 0 || hi >= g->pub.dim[k]))
              return false;
          }
          return true;
        };
        for (int t = 0; t < d.nterms; t++)
          if (!in_bounds(d.terms[t].a) || !in_bounds(d.terms[t].b)) return PSB_ERR_INVALID;
        if (d.has_post && !in_bounds(d.post)) return PSB_ERR_INVALID;
        psb_factor self;
        memset(&self, 0, sizeof(self));
        self.grid = d.out_grid;
        if (!in_bounds(self)) return PSB_ERR_INVALID;
      }
      // A grid that is both read at an offset and written, without
      // red-black ordering, would race; the reference's ref target gives it
      // Gauss-Seidel meaning, which a parallel sweep cannot reproduce.
      if (writes && m.color < 0) {
        const GridImpl *out = m.grids[d.out_grid];
        for (int t = 0; t < d.nterms; t++) {
          const psb_factor *fs[2] = {&d.terms[t].a, &d.terms[t].b};
          for (const psb_factor *f : fs)
            if (f->grid >= 0 && m.grids[f->grid] == out &&
                (f->offset[0] || f->offset[1] || f->offset[2]))
              return PSB_ERR_UNSUPPORTED;
        }
      }
      return PSB_OK;
    }
  }
}

psb_status prepare_ghosts(MapImpl &m) {
  if (m.kernel_id != PSB_KERNEL_DIFFUSION7_PERIODIC) return PSB_OK;
  GridImpl *in = m.grids[0];
  if (in->layout == PSB_LAYOUT_PITCHED && in->ghost_valid != PSB_BOUNDARY_PERIODIC)
    return launch_halo_fill(in, PSB_BOUNDARY_PERIODIC, rt().stream);
  return PSB_OK;
}

// One application of a map on the runtime stream.
psb_status launch_map(MapImpl &m, int color, int64_t *launches) {
  Runtime &r = rt();
  cudaStream_t s = r.stream;
  psb_status st = PSB_OK;
  if (m.kernel_id == PSB_KERNEL_DIFFUSION7 || m.kernel_id == PSB_KERNEL_DIFFUSION7_PERIODIC ||
      m.kernel_id == PSB_KERNEL_HIMENO19) {
    psb_tune_config cfg;
    const int n[3] = {m.grids[0]->pub.dim[0], m.grids[0]->pub.dim[1], m.grids[0]->pub.dim[2]};
    int type = m.grids[0]->pub.elm_size == 8 ? PS_DOUBLE : PS_FLOAT;
    tune_lookup(m.kernel_id, type, n, &cfg);
    if (r.impl == PSB_IMPL_PLAIN) cfg.impl = PSB_IMPL_PLAIN;
    if (r.impl == PSB_IMPL_TMA) cfg.impl = PSB_IMPL_TMA;
    if (m.kernel_id == PSB_KERNEL_HIMENO19)
      st = himeno_launch(m, cfg, s, launches);
    else
      st = diffusion7_launch(m, cfg, s, launches);
    GridImpl *o = m.grids[1];
    if (m.kernel_id != PSB_KERNEL_DIFFUSION7_PERIODIC && o->layout == PSB_LAYOUT_PITCHED)
      o->ghost_valid = PSB_BOUNDARY_NONE;
    // Periodic writers keep the output halo current (images), so a valid
    // halo stays valid; an incomplete domain cannot make it valid.
    if (m.kernel_id == PSB_KERNEL_DIFFUSION7_PERIODIC && o->layout == PSB_LAYOUT_PITCHED) {
      bool full = true;
      for (int i = 0; i < 3; i++)
        if (m.dom.local_min[i] != 0 || m.dom.local_max[i] != o->pub.dim[i]) full = false;
      if (full) o->ghost_valid = PSB_BOUNDARY_PERIODIC;
    }
  } else if (const psb_compiled_stencil *cd = compiled_of(m.kernel_id)) {
    GridImpl *views[PSB_MAX_VIEWS];
    if (compiled_views(m, *cd, views) != cd->nviews) return set_status(PSB_ERR_INVALID);
    psb_launch_args a;
    memset(&a, 0, sizeof(a));
    for (int k = 0; k < 3; k++) {
      a.lo[k] = k < cd->ndims ? m.dom.local_min[k] : 0;
      a.hi[k] = k < cd->ndims ? m.dom.local_max[k] : 1;
    }
    a.color = color;
    a.nviews = cd->nviews;
    a.nparams = m.nparams;
    for (int v = 0; v < cd->nviews; v++) {
      const GridView gv = views[v]->view();
      a.views[v].origin = gv.origin;
      a.views[v].sy = gv.sy;
      a.views[v].sz = gv.sz;
      for (int k = 0; k < 3; k++) a.views[v].n[k] = gv.n[k];
      a.views[v].type = cd->view_type[v];
    }
    for (int i = 0; i < m.nparams; i++) a.params[i] = m.params[i];
    a.error = r.d_error + 1;
    a.device = r.device;
    st = compiled_staged_launch(m, *cd, views, color, s);
    if (st == PSB_ERR_UNSUPPORTED) st = cd->launch(&a, (void *)s);
    if (launches) (*launches)++;
    for (int v = 0; v < cd->nviews; v++)
      if (cd->view_emits[v] && views[v]->layout == PSB_LAYOUT_PITCHED)
        views[v]->ghost_valid = PSB_BOUNDARY_NONE;
  } else {
    const GenericDesc *gd = generic_of(m.kernel_id);
    if (!gd) return set_status(PSB_ERR_INVALID);
    st = generic_launch(m, *gd, color, s, launches);
    GridImpl *o = m.grids[gd->host.out_grid];
    if (o->layout == PSB_LAYOUT_PITCHED) o->ghost_valid = PSB_BOUNDARY_NONE;
  }
  if (st != PSB_OK) return st;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "kernel launch");
  return PSB_OK;
}

// Launch every map of one iteration (red-black maps twice).
static psb_status launch_iteration(MapImpl **ms, int n, int64_t *launches) {
  for (int i = 0; i < n; i++) {
    MapImpl &m = *ms[i];
    if (m.color == 2) {
      PSB_CHECK(launch_map(m, 0, launches));
      PSB_CHECK(launch_map(m, 1, launches));
    } else {
      PSB_CHECK(launch_map(m, m.color, launches));
    }
  }
  return PSB_OK;
}

static std::string graph_key(MapImpl **ms, int n, int unroll) {
  // Maps are identified by their slot; a slot is only reused after
  // psb_stencil_free, which drops every cached graph.
  std::string k = std::to_string(unroll) + ":";
  for (int i = 0; i < n; i++) k += std::to_string(ms[i] - rt().maps.data()) + ",";
  return k;
}

static void drop_graphs() {
  for (auto &kv : rt().graphs) cudaGraphExecDestroy(kv.second);
  rt().graphs.clear();
}
void drop_all_graphs() { drop_graphs(); }

// A freed grid ends every map that binds it (its handle becomes invalid).
void maps_forget_grid(const GridImpl *g) {
  for (auto &m : rt().maps) {
    if (!m.live) continue;
    bool uses = false;
    for (int i = 0; i < m.ngrids; i++) uses = uses || m.grids[i] == g;
    if (!uses) continue;
    if (m.d_partials) cudaFree(m.d_partials);
    if (m.d_ticket) cudaFree(m.d_ticket);
    if (m.d_history) cudaFree(m.d_history);
    m = MapImpl();
  }
}

// The pattern temporal blocking applies to: PSStencilRun(m1, m2, iter) with
// m1: A -> B and m2: B -> A the same clamped float 7-point map over the
// whole of two pitched grids.
static bool tb2_pair(MapImpl **ms, int n) {
  if (n != 2) return false;
  const MapImpl &a = *ms[0], &b = *ms[1];
  if (a.kernel_id != PSB_KERNEL_DIFFUSION7 || b.kernel_id != PSB_KERNEL_DIFFUSION7) return false;
  if (a.color != -1 || b.color != -1 || a.nparams != 7 || b.nparams != 7) return false;
  for (int i = 0; i < 7; i++)
    if (a.params[i] != b.params[i]) return false;
  GridImpl *A = a.grids[0], *B = a.grids[1];
  if (b.grids[0] != B || b.grids[1] != A || A == B) return false;
  for (GridImpl *g : {A, B}) {
    if (g->layout != PSB_LAYOUT_PITCHED || g->type != PS_FLOAT || g->pub.num_dims != 3 ||
        !tma_eligible(g))
      return false;
    for (int i = 0; i < 3; i++)
      if (g->pub.dim[i] != A->pub.dim[i]) return false;
  }
  for (const MapImpl *m : {&a, &b})
    for (int i = 0; i < 3; i++)
      if (m->dom.local_min[i] != 0 || m->dom.local_max[i] != A->pub.dim[i]) return false;
  return true;
}

// iter pairs as F two-step launches (F the largest even number below iter)
// alternating A -> B and B -> A, then the remaining one or two pairs
// unfused: both grids end exactly as after the unfused run (A the last
// step, B the one before it).
static psb_status run_tb2(MapImpl **ms, int iter, int zchunk, int64_t *launches) {
  Runtime &r = rt();
  GridImpl *A = ms[0]->grids[0], *B = ms[0]->grids[1];
  const int F = (iter - 1) & ~1;
  for (int f = 0; f < F; f++)
    PSB_CHECK(diffusion7_tb2_launch(*ms[0], f & 1 ? B : A, f & 1 ? A : B, zchunk, r.stream,
                                    launches));
  A->ghost_valid = B->ghost_valid = PSB_BOUNDARY_NONE;
  for (int it = F; it < iter; it++) PSB_CHECK(launch_iteration(ms, 2, launches));
  return PSB_OK;
}

// The same for a Himeno pair (two sweeps per launch, k_himeno_tb2.cu): each
// launch runs m1's sweep then m2's, alternating A -> B and B -> A.
static psb_status run_himeno_tb2(MapImpl **ms, int iter, int zchunk, int64_t *launches) {
  Runtime &r = rt();
  GridImpl *A = ms[0]->grids[0], *B = ms[0]->grids[1];
  const int F = (iter - 1) & ~1;
  for (int f = 0; f < F; f++)
    PSB_CHECK(himeno_tb2_launch(*ms[0], *ms[1], f & 1 ? B : A, f & 1 ? A : B, zchunk, r.stream,
                                launches));
  for (int it = F; it < iter; it++) PSB_CHECK(launch_iteration(ms, 2, launches));
  return PSB_OK;
}

static psb_status run_maps(MapImpl **ms, int n, int iter) {
  Runtime &r = rt();
  if (iter <= 0) return PSB_OK;
  for (int i = 0; i < n; i++) PSB_CHECK(check_map(*ms[i]));
  for (int i = 0; i < n; i++) PSB_CHECK(prepare_ghosts(*ms[i]));
  int64_t launches = 0;
  legacy_join_in();
  PSB_TRY(cudaEventRecord(r.ev_start, r.stream));
  if (r.impl != PSB_IMPL_PLAIN && r.impl != PSB_IMPL_GENERIC && tb2_pair(ms, n)) {
    psb_tune_config cfg;
    const int *dims = ms[0]->grids[0]->pub.dim;
    tune_lookup(PSB_KERNEL_DIFFUSION7, PS_FLOAT, dims, &cfg);
    if (cfg.t_depth == 2) {
      PSB_CHECK(run_tb2(ms, iter, cfg.z_chunk, &launches));
      PSB_TRY(cudaEventRecord(r.ev_stop, r.stream));
      legacy_join_out();
      r.last_launches = launches;
      r.last_timed = true;
      return PSB_OK;
    }
  }
  if (r.impl != PSB_IMPL_PLAIN && r.impl != PSB_IMPL_GENERIC && himeno_tb2_pair(ms, n) &&
      iter >= 3) {
    psb_tune_config cfg;
    const int *dims = ms[0]->grids[0]->pub.dim;
    tune_lookup(PSB_KERNEL_HIMENO19, PS_FLOAT, dims, &cfg);
    if (cfg.t_depth == 2) {
      PSB_CHECK(run_himeno_tb2(ms, iter, cfg.z_chunk, &launches));
      PSB_TRY(cudaEventRecord(r.ev_stop, r.stream));
      legacy_join_out();
      r.last_launches = launches;
      r.last_timed = true;
      return PSB_OK;
    }
  }
  // The first iteration always runs eagerly: it performs every lazy set-up
  // (TMA descriptors, residual buffers, kernel attributes) outside stream
  // capture. The remaining iterations replay a CUDA graph of `unroll`
  // iterations.
  PSB_CHECK(launch_iteration(ms, n, &launches));
  int rest = iter - 1;
  const bool graph = r.use_graph && rest >= 2;
  if (!graph) {
    for (int it = 0; it < rest; it++) PSB_CHECK(launch_iteration(ms, n, &launches));
  } else {
    const int unroll = std::min(rest, kUnroll);
    std::string key = graph_key(ms, n, unroll);
    cudaGraphExec_t exec = nullptr;
    auto it = r.graphs.find(key);
    // Kernel arguments (tensor maps, pointers) are baked into the graph;
    // they only change when grids or maps are freed or the tuning changes,
    // which drops all graphs.
    if (it != r.graphs.end()) exec = it->second;
    int64_t per_iter = 0;
    for (int i = 0; i < n; i++) per_iter += ms[i]->color == 2 ? 2 : 1;
    if (!exec) {
      cudaGraph_t g;
      PSB_TRY(cudaStreamBeginCapture(r.stream, cudaStreamCaptureModeThreadLocal));
      int64_t dummy = 0;
      psb_status st = PSB_OK;
      for (int u = 0; u < unroll && st == PSB_OK; u++) st = launch_iteration(ms, n, &dummy);
      cudaError_t e = cudaStreamEndCapture(r.stream, &g);
      if (st != PSB_OK || e != cudaSuccess) {
        if (e == cudaSuccess) cudaGraphDestroy(g);
        cudaGetLastError();  // do not leave a capture error for later calls
        return st != PSB_OK ? set_status(st) : cuda_status(e, "cudaStreamEndCapture");
      }
      e = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_status(e, "cudaGraphInstantiate");
      }
      r.graphs[key] = exec;
    }
    const int reps = rest / unroll;
    for (int k = 0; k < reps; k++) {
      PSB_TRY(cudaGraphLaunch(exec, r.stream));
      launches += per_iter * unroll;
    }
    for (int k = 0; k < rest % unroll; k++) PSB_CHECK(launch_iteration(ms, n, &launches));
  }
  PSB_TRY(cudaEventRecord(r.ev_stop, r.stream));
  legacy_join_out();
  r.last_launches = launches;
  r.last_timed = true;
  if (__ps_trace) {
    float ms_ = 0;
    cudaEventSynchronize(r.ev_stop);
    cudaEventElapsedTime(&ms_, r.ev_start, r.ev_stop);
    fprintf(__ps_trace, "Physis: Stencil finished (time: %f)\n", ms_);
  }
  return PSB_OK;
}

static psb_status make_map(int kernel_id, const __PSDomain *dom, __PSGrid *const *grids,
                           int ngrids, const double *params, int nparams, int color,
                           PSStencil *out) {
  PSB_CHECK(ensure_init());
  if (!dom || !out || ngrids < 1 || ngrids > PSB_MAX_GRIDS || nparams < 0 ||
      nparams > PSB_MAX_PARAMS)
    return set_status(PSB_ERR_INVALID);
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  MapImpl m;
  m.kernel_id = kernel_id;
  m.dom = *dom;
  m.ngrids = ngrids;
  // A grid of a point type (psb_grid_new_user) has no storage of its own:
  // only compiled stencils bind it whole (other kernels take components).
  const bool compiled = compiled_of(kernel_id) != nullptr;
  for (int i = 0; i < ngrids; i++) {
    m.grids[i] = as_impl(grids[i]);
    if (!m.grids[i] || m.grids[i]->user_type || (!m.grids[i]->comps.empty() && !compiled))
      return set_status(PSB_ERR_INVALID);
  }
  m.nparams = nparams;
  for (int i = 0; i < nparams; i++) m.params[i] = params[i];
  m.color = color;
  m.live = true;
  PSB_CHECK(check_map(m));
  // The same closure bound again (a map call inside the user's time loop)
  // returns the existing handle instead of growing the table.
  for (int i = 0; i < (int)r.maps.size(); i++) {
    const MapImpl &o = r.maps[i];
    if (!o.live || o.kernel_id != m.kernel_id || o.ngrids != m.ngrids ||
        o.nparams != m.nparams || o.color != m.color ||
        memcmp(&o.dom, &m.dom, sizeof(m.dom)) != 0)
      continue;
    bool same = true;
    for (int k = 0; k < m.ngrids; k++) same = same && o.grids[k] == m.grids[k];
    for (int k = 0; k < m.nparams; k++) same = same && o.params[k] == m.params[k];
    if (same && o.residual_len == 0) {
      *out = kHandleTag | i;
      return PSB_OK;
    }
  }
  int idx = -1;
  for (int i = 0; i < (int)r.maps.size(); i++)
    if (!r.maps[i].live && !r.maps[i].d_partials) {
      idx = i;
      break;
    }
  if (idx < 0) {
    idx = (int)r.maps.size();
    r.maps.push_back(m);
  } else {
    r.maps[idx] = m;
  }
  *out = kHandleTag | idx;
  return PSB_OK;
}

// Number of grid arguments a kernel takes through PSStencilMap varargs.
static int kernel_ngrids(int kernel_id, int *nparams) {
  switch (kernel_id) {
    case PSB_KERNEL_DIFFUSION7:
    case PSB_KERNEL_DIFFUSION7_PERIODIC: *nparams = 7; return 2;
    case PSB_KERNEL_HIMENO19: *nparams = 1; return 14;
    default: {
      if (const psb_compiled_stencil *cd = compiled_of(kernel_id)) {
        *nparams = cd->nparams;
        return cd->ngrids;
      }
      const GenericDesc *gd = generic_of(kernel_id);
      *nparams = 0;
      return gd ? gd->host.ngrids : -1;
    }
  }
}

static PSStencil vmap(void *kernel, int color, va_list vl) {
  std::unique_lock<std::recursive_mutex> lk(rt().mu);
  int kid = (int)(intptr_t)kernel;
  int np = 0;
  int ng = kernel_ngrids(kid, &np);
  if (ng < 0) {
    lk.unlock();
    fprintf(stderr, "physis_b200: PSStencilMap: unknown kernel %d\n", kid);
    exit(EXIT_FAILURE);
  }
  __PSDomain dom = va_arg(vl, __PSDomain);
  __PSGrid *grids[PSB_MAX_GRIDS];
  for (int i = 0; i < ng; i++) grids[i] = va_arg(vl, __PSGrid *);
  double params[PSB_MAX_PARAMS];
  // Varargs promote float to double; integer scalars of compiled stencils
  // arrive as int / long.
  const psb_compiled_stencil *cd = compiled_of(kid);
  for (int i = 0; i < np; i++) {
    const int t = cd ? cd->param_type[i] : PS_DOUBLE;
    if (t == PS_INT)
      params[i] = (double)va_arg(vl, int);
    else if (t == PS_LONG)
      params[i] = (double)va_arg(vl, long);
    else
      params[i] = va_arg(vl, double);
  }
  PSStencil h = 0;
  psb_status s = make_map(kid, &dom, grids, ng, params, np, color, &h);
  lk.unlock();
  if (s != PSB_OK) {
    fprintf(stderr, "physis_b200: PSStencilMap failed: %s\n", psb_status_string(s));
    exit(EXIT_FAILURE);
  }
  return h;
}

psb_status fetch_history(MapImpl &m, double *out, int n) {
  if (m.residual_len <= 0 || !m.d_history) return set_status(PSB_ERR_INVALID);
  PSB_TRY(cudaStreamSynchronize(rt().stream));
  unsigned count = 0;
  PSB_TRY(cudaMemcpy(&count, m.d_counter, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (count == 0) return set_status(PSB_ERR_INVALID);
  std::vector<double> h(m.residual_len);
  PSB_TRY(cudaMemcpy(h.data(), m.d_history, sizeof(double) * m.residual_len,
                     cudaMemcpyDeviceToHost));
  // Most recent last.
  for (int i = 0; i < n; i++) {
    int64_t k = (int64_t)count - n + i;
    out[i] = k < 0 ? 0.0 : h[k % m.residual_len];
  }
  return PSB_OK;
}

}  // namespace psb

using namespace psb;

extern "C" {

PSStencil __PSStencilMap(void *kernel, ...) {
  va_list vl;
  va_start(vl, kernel);
  PSStencil h = vmap(kernel, -1, vl);
  va_end(vl);
  return h;
}
PSStencil __PSStencilMapRedBlack(void *kernel, ...) {
  va_list vl;
  va_start(vl, kernel);
  PSStencil h = vmap(kernel, 2, vl);
  va_end(vl);
  return h;
}
PSStencil __PSStencilMapRed(void *kernel, ...) {
  va_list vl;
  va_start(vl, kernel);
  PSStencil h = vmap(kernel, 0, vl);
  va_end(vl);
  return h;
}
PSStencil __PSStencilMapBlack(void *kernel, ...) {
  va_list vl;
  va_start(vl, kernel);
  PSStencil h = vmap(kernel, 1, vl);
  va_end(vl);
  return h;
}

void __PSStencilRunN(int nargs, ...) {
  va_list vl;
  va_start(vl, nargs);
  PSStencil hs[PSB_B200_MAX_RUN_MAPS];
  int nm = 0, iter = 1;
  std::unique_lock<std::recursive_mutex> lk(rt().mu);
  for (int i = 0; i < nargs; i++) {
    int v = va_arg(vl, int);
    if (map_of(v) && nm < PSB_B200_MAX_RUN_MAPS) {
      hs[nm++] = v;
    } else if (i == nargs - 1) {
      iter = v;
    } else {
      lk.unlock();
      fprintf(stderr, "physis_b200: PSStencilRun: argument %d is not a stencil map\n", i);
      exit(EXIT_FAILURE);
    }
  }
  va_end(vl);
  psb_status s = psb_stencil_run(hs, nm, iter);
  lk.unlock();
  if (s != PSB_OK) {
    fprintf(stderr, "physis_b200: PSStencilRun failed: %s\n", psb_status_string(s));
    exit(EXIT_FAILURE);
  }
}

psb_status psb_generic_register(const psb_generic_stencil *desc, int *kernel_id) {
  PSB_CHECK(ensure_init());
  if (!desc || !kernel_id) return set_status(PSB_ERR_INVALID);
  const psb_generic_stencil &d = *desc;
  if (d.ndims < 1 || d.ndims > 3 || d.ngrids < 1 || d.ngrids > PSB_MAX_GRIDS || d.nterms < 1 ||
      d.nterms > PSB_MAX_TERMS || d.out_grid < 0 || d.out_grid >= d.ngrids)
    return set_status(PSB_ERR_INVALID);
  if (type_size(d.accum_type) == 0) return set_status(PSB_ERR_INVALID);
  auto check_factor = [&](const psb_factor &f) {
    if (f.grid >= d.ngrids) return false;
    if (f.boundary < 0 || f.boundary > 2) return false;
    return true;
  };
  for (int i = 0; i < d.ngrids; i++) {
    if (type_size(d.grid_type[i]) == 0) return set_status(PSB_ERR_INVALID);
    for (int k = 0; k < 3; k++)
      if (d.grid_axes[i][k] >= d.ndims) return set_status(PSB_ERR_INVALID);
  }
  for (int t = 0; t < d.nterms; t++)
    if (!check_factor(d.terms[t].a) || !check_factor(d.terms[t].b))
      return set_status(PSB_ERR_INVALID);
  if (d.has_post && !check_factor(d.post)) return set_status(PSB_ERR_INVALID);
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  GenericDesc gd;
  gd.host = d;
  PSB_CHECK(generic_upload(gd));
  r.generics.push_back(gd);
  *kernel_id = PSB_KERNEL_FIRST_GENERIC + (int)r.generics.size() - 1;
  return PSB_OK;
}

psb_status psb_stencil_map(int kernel_id, const __PSDomain *dom, __PSGrid *const *grids,
                           int ngrids, const double *params, int nparams, PSStencil *out) {
  return make_map(kernel_id, dom, grids, ngrids, params, nparams, -1, out);
}

psb_status psb_compiled_register(const psb_compiled_stencil *desc, int *kernel_id) {
  PSB_CHECK(ensure_init());
  if (!desc || !kernel_id || !desc->launch) return set_status(PSB_ERR_INVALID);
  const psb_compiled_stencil &d = *desc;
  if (d.ndims < 1 || d.ndims > 3 || d.ngrids < 1 || d.ngrids > PSB_MAX_GRIDS || d.nparams < 0 ||
      d.nparams > PSB_MAX_PARAMS)
    return set_status(PSB_ERR_INVALID);
  int nv = 0;
  for (int i = 0; i < d.ngrids; i++) {
    const bool user = d.grid_type[i] == PS_USER;
    if ((!user && (type_size(d.grid_type[i]) == 0 || d.grid_components[i] != 1)) ||
        d.grid_components[i] < 1 || d.grid_ndims[i] < 1 || d.grid_ndims[i] > 3)
      return set_status(PSB_ERR_INVALID);
    nv += d.grid_components[i];
  }
  if (nv != d.nviews || nv > PSB_MAX_VIEWS) return set_status(PSB_ERR_INVALID);
  for (int v = 0; v < d.nviews; v++)
    if (type_size(d.view_type[v]) == 0) return set_status(PSB_ERR_INVALID);
  for (int i = 0; i < d.nparams; i++)
    if (type_size(d.param_type[i]) == 0) return set_status(PSB_ERR_INVALID);
  if (d.staged_checked && !d.staged) return set_status(PSB_ERR_INVALID);
  if (d.staged) {
    if ((d.staged_type != PS_FLOAT && d.staged_type != PS_DOUBLE) || d.ndims != 3 ||
        d.staged_emit < 0 || d.staged_emit >= d.ngrids)
      return set_status(PSB_ERR_INVALID);
    for (int i = 0; i < d.ngrids; i++) {
      if (d.grid_type[i] != d.staged_type || d.grid_ndims[i] != 3)
        return set_status(PSB_ERR_INVALID);
      if (d.read_lo[i][0] > d.read_hi[i][0]) {  // not read
        if (d.read_periodic[i]) return set_status(PSB_ERR_INVALID);
        continue;
      }
      if (i == d.staged_emit) return set_status(PSB_ERR_INVALID);
      for (int k = 0; k < 3; k++)
        if (d.read_lo[i][k] < -2 || d.read_hi[i][k] > 2 || d.read_lo[i][k] > d.read_hi[i][k])
          return set_status(PSB_ERR_INVALID);
    }
  }
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  r.compiled.push_back(d);
  *kernel_id = PSB_KERNEL_FIRST_COMPILED + (int)r.compiled.size() - 1;
  return PSB_OK;
}

psb_status psb_stencil_map_rb(int kernel_id, const __PSDomain *dom, __PSGrid *const *grids,
                              int ngrids, const double *params, int nparams, int color,
                              PSStencil *out) {
  if (color < 0 || color > 2) return set_status(PSB_ERR_INVALID);
  std::lock_guard<std::recursive_mutex> lk(rt().mu);
  if (!generic_of(kernel_id) && !compiled_of(kernel_id)) return set_status(PSB_ERR_UNSUPPORTED);
  return make_map(kernel_id, dom, grids, ngrids, params, nparams, color, out);
}

psb_status psb_stencil_run(const PSStencil *maps, int nmaps, int iter) {
  PSB_CHECK(ensure_init());
  if (nmaps < 1 || nmaps > PSB_B200_MAX_RUN_MAPS || !maps) return set_status(PSB_ERR_INVALID);
  // Map and kernel tables grow under the runtime lock; entries are only
  // looked up and used while holding it.
  std::lock_guard<std::recursive_mutex> lk(rt().mu);
  MapImpl *ms[PSB_B200_MAX_RUN_MAPS];
  for (int i = 0; i < nmaps; i++) {
    ms[i] = map_of(maps[i]);
    if (!ms[i]) return set_status(PSB_ERR_INVALID);
  }
  return run_maps(ms, nmaps, iter);
}

psb_status psb_stencil_free(PSStencil s) {
  std::lock_guard<std::recursive_mutex> lk(rt().mu);
  MapImpl *m = map_of(s);
  if (!m) return set_status(PSB_ERR_INVALID);
  cudaStreamSynchronize(rt().stream);
  drop_graphs();
  if (m->d_partials) cudaFree(m->d_partials);
  if (m->d_ticket) cudaFree(m->d_ticket);
  // d_counter points into the d_ticket allocation.
  if (m->d_history) cudaFree(m->d_history);
  *m = MapImpl();
  return PSB_OK;
}

psb_status psb_set_impl(int impl) {
  if (impl < PSB_IMPL_AUTO || impl > PSB_IMPL_GENERIC) return set_status(PSB_ERR_INVALID);
  PSB_CHECK(ensure_init());
  rt().impl = impl;
  drop_graphs();
  return PSB_OK;
}

psb_status psb_set_fp_mode(int mode) {
  if (mode != PSB_FP_EXACT && mode != PSB_FP_FMA) return set_status(PSB_ERR_INVALID);
  PSB_CHECK(ensure_init());
  rt().fp_mode = mode;
  drop_graphs();
  return PSB_OK;
}

psb_status psb_get_fp_mode(int *mode) {
  if (!mode) return set_status(PSB_ERR_INVALID);
  PSB_CHECK(ensure_init());
  *mode = rt().fp_mode;
  return PSB_OK;
}

psb_status psb_set_graph(int enable) {
  PSB_CHECK(ensure_init());
  rt().use_graph = enable != 0;
  return PSB_OK;
}

psb_status psb_himeno_residual_enable(PSStencil h, int history_len) {
  std::lock_guard<std::recursive_mutex> lk(rt().mu);
  MapImpl *m = map_of(h);
  if (!m || m->kernel_id != PSB_KERNEL_HIMENO19 || history_len < 0)
    return set_status(PSB_ERR_INVALID);
  drop_graphs();
  if (history_len == 0) {
    m->residual_len = 0;
    return PSB_OK;
  }
  if (!m->d_ticket) {
    PSB_TRY(cudaMalloc(&m->d_ticket, sizeof(unsigned) * 2));
    m->d_counter = m->d_ticket + 1;
  }
  PSB_TRY(cudaMemset(m->d_ticket, 0, sizeof(unsigned) * 2));
  if (m->d_history) cudaFree(m->d_history);
  m->d_history = nullptr;
  PSB_TRY(cudaMalloc(&m->d_history, sizeof(double) * history_len));
  PSB_TRY(cudaMemset(m->d_history, 0, sizeof(double) * history_len));
  m->residual_len = history_len;
  return PSB_OK;
}

psb_status psb_himeno_residual(PSStencil h, double *gosa) {
  std::lock_guard<std::recursive_mutex> lk(rt().mu);
  MapImpl *m = map_of(h);
  if (!m || !gosa) return set_status(PSB_ERR_INVALID);
  return fetch_history(*m, gosa, 1);
}

psb_status psb_himeno_residual_history(PSStencil h, double *out, int n) {
  std::lock_guard<std::recursive_mutex> lk(rt().mu);
  MapImpl *m = map_of(h);
  if (!m || !out || n < 1 || n > m->residual_len) return set_status(PSB_ERR_INVALID);
  return fetch_history(*m, out, n);
}

psb_status psb_last_run_stats(double *device_ms, int64_t *launches) {
  Runtime &r = rt();
  if (!r.last_timed) return set_status(PSB_ERR_INVALID);
  PSB_TRY(cudaEventSynchronize(r.ev_stop));
  float ms = 0;
  PSB_TRY(cudaEventElapsedTime(&ms, r.ev_start, r.ev_stop));
  if (device_ms) *device_ms = ms;
  if (launches) *launches = r.last_launches;
  return PSB_OK;
}

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------

static psb_status reduce_grid(GridImpl *g, int type, int op, const __PSDomain *dom, double *res) {
  if (!g || g->user_type || !g->comps.empty() || op < PS_MAX || op > PS_PROD)
    return set_status(PSB_ERR_INVALID);
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    const int n = i < g->pub.num_dims ? g->pub.dim[i] : 1;
    d.lo[i] = dom && i < g->pub.num_dims ? dom->local_min[i] : 0;
    d.hi[i] = dom && i < g->pub.num_dims ? dom->local_max[i] : n;
    if (d.lo[i] < 0 || d.hi[i] > n || d.hi[i] <= d.lo[i]) return set_status(PSB_ERR_INVALID);
  }
  GridView v = g->view();
  legacy_join_in();
  return reduce_view(v, type, op, d, res, rt().stream);
}

}  // extern "C"

namespace {
template <typename T>
void reduce_abi(void *buf, enum PSReduceOp op, __PSGrid *p, int type) {
  GridImpl *g = as_impl(p);
  double r = 0;
  psb_status s = g ? reduce_grid(g, type, (int)op, nullptr, &r) : PSB_ERR_INVALID;
  if (s != PSB_OK) {
    fprintf(stderr, "physis_b200: PSReduce failed: %s\n", psb_status_string(s));
    exit(EXIT_FAILURE);
  }
  *(T *)buf = (T)r;
}
}  // namespace

extern "C" {

void __PSReduceGridFloat(void *buf, enum PSReduceOp op, __PSGrid *g) {
  reduce_abi<float>(buf, op, g, PS_FLOAT);
}

void __PSReduceGridDouble(void *buf, enum PSReduceOp op, __PSGrid *g) {
  reduce_abi<double>(buf, op, g, PS_DOUBLE);
}

void(PSReduce)(void *v, ...) {
  // PSReduce(&v, op, grid): the grid form of physis_user.h:114. The result
  // type follows the grid's element type.
  va_list vl;
  va_start(vl, v);
  int op = va_arg(vl, int);
  __PSGrid *p = va_arg(vl, __PSGrid *);
  va_end(vl);
  GridImpl *g = as_impl(p);
  if (!g) {
    fprintf(stderr, "physis_b200: PSReduce: not a grid\n");
    exit(EXIT_FAILURE);
  }
  switch (g->type) {
    case PS_DOUBLE: reduce_abi<double>(v, (PSReduceOp)op, p, PS_DOUBLE); break;
    case PS_INT: reduce_abi<int32_t>(v, (PSReduceOp)op, p, PS_INT); break;
    case PS_LONG: reduce_abi<int64_t>(v, (PSReduceOp)op, p, PS_LONG); break;
    default: reduce_abi<float>(v, (PSReduceOp)op, p, PS_FLOAT); break;
  }
}

psb_status psb_reduce_map(int kernel_id, const __PSDomain *dom, __PSGrid *const *grids,
                          int ngrids, const double *params, int nparams, int op,
                          double *result) {
  PSB_CHECK(ensure_init());
  if (!dom || !grids || !result || op < PS_MAX || op > PS_PROD || ngrids < 1 ||
      ngrids > PSB_MAX_GRIDS || nparams < 0 || nparams > PSB_MAX_PARAMS)
    return set_status(PSB_ERR_INVALID);
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  const GenericDesc *gd = generic_of(kernel_id);
  if (!gd) return set_status(kernel_id < PSB_KERNEL_FIRST_GENERIC ? PSB_ERR_UNSUPPORTED
                                                                  : PSB_ERR_INVALID);
  MapImpl m;
  m.kernel_id = kernel_id;
  m.dom = *dom;
  m.ngrids = ngrids;
  for (int i = 0; i < ngrids; i++) {
    m.grids[i] = as_impl(grids[i]);
    if (!m.grids[i] || m.grids[i]->user_type || !m.grids[i]->comps.empty())
      return set_status(PSB_ERR_INVALID);
  }
  m.nparams = nparams;
  for (int i = 0; i < nparams; i++) m.params[i] = params[i];
  PSB_CHECK(check_map(m, false));
  legacy_join_in();
  PSB_CHECK(generic_reduce(m, *gd, op, result, r.stream));
  legacy_join_out();
  return PSB_OK;
}

// PSReduce(&v, op, grid) or PSReduce(&v, op, kernel, dom, grids...): the
// macro passes the argument count. The kernel form reduces the values the
// stencil would emit; v has the emitted grid's element type.
void __PSReduceN(int nargs, void *v, ...) {
  va_list vl;
  va_start(vl, v);
  const int op = va_arg(vl, int);
  if (nargs == 3) {
    __PSGrid *g = va_arg(vl, __PSGrid *);
    va_end(vl);
    (PSReduce)(v, op, g);
    return;
  }
  const int kid = (int)(intptr_t)va_arg(vl, void *);
  int np = 0;
  const int ng = kernel_ngrids(kid, &np);
  if (ng < 0) {
    va_end(vl);
    fprintf(stderr, "physis_b200: PSReduce: unknown kernel %d\n", kid);
    exit(EXIT_FAILURE);
  }
  __PSDomain dom = va_arg(vl, __PSDomain);
  __PSGrid *grids[PSB_MAX_GRIDS];
  for (int i = 0; i < ng; i++) grids[i] = va_arg(vl, __PSGrid *);
  va_end(vl);
  double r = 0;
  psb_status s = psb_reduce_map(kid, &dom, grids, ng, nullptr, 0, op, &r);
  if (s != PSB_OK) {
    fprintf(stderr, "physis_b200: PSReduce failed: %s\n", psb_status_string(s));
    exit(EXIT_FAILURE);
  }
  const GenericDesc *gd = generic_of(kid);
  switch (gd->host.grid_type[gd->host.out_grid]) {
    case PS_DOUBLE: *(double *)v = r; break;
    case PS_INT: *(int32_t *)v = (int32_t)r; break;
    case PS_LONG: *(int64_t *)v = (int64_t)r; break;
    default: *(float *)v = (float)r; break;
  }
}

psb_status psb_reduce(__PSGrid *p, int op, const __PSDomain *dom, double *result) {
  PSB_CHECK(ensure_init());
  GridImpl *g = as_impl(p);
  if (!g || !result) return set_status(PSB_ERR_INVALID);
  int type = g->type >= 0 ? g->type : type_from_size(g->pub.elm_size);
  return reduce_grid(g, type, op, dom, result);
}

}  // extern "C"
