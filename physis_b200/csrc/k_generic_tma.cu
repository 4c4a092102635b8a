// Generic flat linear stencil on the TMA plane pipeline (2.5-D z-streaming).
//
// The B200 path for user stencils registered as psb_generic_stencil (the
// executable form of the reference's flat-sum stencil functions,
// tests/system_tests/test_cases/test_*.c, which its CUDA target turns into
// one-thread-per-(x,y) kernels with a z loop and global loads,
// translator/cuda_translator.cc:615-869). Here each CTA owns a TX x TY
// column of the domain and a chunk of z. A producer thread streams, for
// every input plane, one TMA box of each grid the stencil reads -- the tile
// plus the halo the term table's offsets need (|offset| <= 2 per axis) --
// into a ring of shared-memory stages; the z offsets of the table set how
// many planes are live at once (a window of zmax - zmin + 1 stages), so
// every input plane is read from HBM once per tile. Consumer warps evaluate
// the term table on the staged planes: each thread owns V consecutive x
// points (16 bytes) of VY rows, reads every factor from shared memory and
// stores 16 bytes at a time.
//
// Arithmetic and order are those of k_generic (and of the reference's CPU
// target): each term a_i * b_i rounded in the accumulation type, summed left
// to right, times the optional post factor; a factor that is the constant 1
// is not multiplied (x * 1 == x exactly). Results are bit-identical to the
// thread-per-point kernel.
//
// Boundary forms: plain reads take the grid's own cells (the map was checked
// to stay inside the grid); periodic and clamped reads take the resident
// halo of a pitched grid, which the launcher refreshes with the periodic or
// clamped image of the interior (k_halo_fill) whenever the grid changed
// since. A grid read both ways, an in-place map, red-black order, lower-
// dimensional or mixed-type grids, and offsets beyond the halo use k_generic.
#include <algorithm>
#include <cstring>

#include "k_generic.cuh"
#include "k_generic_tma.cuh"

namespace psb {

template <typename T>
__global__ void __launch_bounds__(kGtThreads, sizeof(T) == 4 ? 4 : 3)
    k_generic_tma(const __grid_constant__ GtMaps maps, const __grid_constant__ GtTable tab,
                  GridView out, Dom3 d, const __grid_constant__ GtGeom geo, int *err) {
  gt_body<T, GtTableProg>(maps, tab, out, d, geo, err);
}

// Host: decide whether the map runs on the TMA path and build its table.
struct GtPlan {
  int ngrids = 0;
  int slots[kGtMaxGrids];     // stencil grid slot of each staged grid
  int mode[kGtMaxGrids];      // halo form each staged grid needs (NONE: none)
  int zmin = 0, zmax = 0;
};

static bool gt_factor_ok(const psb_generic_stencil &d, const MapImpl &m, const psb_factor &f,
                         GtPlan &p) {
  if (f.grid < 0) return true;
  if (f.grid >= d.ngrids || f.grid == d.out_grid) return false;
  if (d.grid_type[f.grid] != d.accum_type) return false;
  for (int k = 0; k < 3; k++)
    if (d.grid_axes[f.grid][k] != k || f.offset[k] < -kGtR || f.offset[k] > kGtR) return false;
  if (m.grids[f.grid] == m.grids[d.out_grid]) return false;  // in place
  int gi = -1;
  for (int i = 0; i < p.ngrids; i++)
    if (p.slots[i] == f.grid) gi = i;
  if (gi < 0) {
    if (p.ngrids == kGtMaxGrids) return false;
    gi = p.ngrids++;
    p.slots[gi] = f.grid;
    p.mode[gi] = PSB_BOUNDARY_NONE;
  }
  if (f.boundary != PSB_BOUNDARY_NONE) {
    if (p.mode[gi] != PSB_BOUNDARY_NONE && p.mode[gi] != f.boundary) return false;
    if (m.grids[f.grid]->layout != PSB_LAYOUT_PITCHED) return false;
    p.mode[gi] = f.boundary;
  }
  p.zmin = std::min(p.zmin, f.offset[2]);
  p.zmax = std::max(p.zmax, f.offset[2]);
  return true;
}

static GtFactor gt_compact(const psb_factor &f, const GtPlan &p, int plane_elems, int bx) {
  GtFactor g;
  memset(&g, 0, sizeof(g));
  if (f.grid < 0) {
    g.kind = f.constant == 1.0 ? 1 : 0;
    g.c = f.constant;
    return g;
  }
  int gi = 0;
  for (int i = 0; i < p.ngrids; i++)
    if (p.slots[i] == f.grid) gi = i;
  g.kind = 2;
  g.k = f.offset[2] - p.zmin;
  g.off = gi * plane_elems + f.offset[1] * bx + f.offset[0];
  return g;
}

static int g_last_generic_impl = PSB_IMPL_GENERIC;
static int g_last_generic_compiled = 0;
static int g_generic_compile = -1;  // -1: $PHYSIS_B200_GENERIC_COMPILE (default on)

static bool generic_compile_on() {
  if (g_generic_compile < 0) {
    const char *e = getenv("PHYSIS_B200_GENERIC_COMPILE");
    g_generic_compile = e && e[0] == '0' ? 0 : 1;
  }
  return g_generic_compile == 1;
}

// Source of a kernel for one table, the library's device headers plus its
// term program written out with every structural field as a constant.
// Packed tables: which rows to load and when, which neighbouring lanes each
// run needs, each term's x offset and whether it is multiplied (the program
// GtTableProg interprets word by word). General tables: each factor's kind,
// window plane and offset (the loop the interpreting kernel runs).
// Coefficients stay in the launch's table (read at constant offsets), so
// tables that differ only in coefficients share one kernel.
static std::string gt_factor_src(const GtFactor &f, const char *side, int t) {
  return "GtFactor{" + std::to_string(f.kind) + ", " + std::to_string(f.k) + ", " +
         std::to_string(f.off) + ", 0, tab." + side + "[" + std::to_string(t) + "].c}";
}

static std::string gt_jit_source(const GtTable &tab, bool dbl, bool fma, std::string *key) {
  const char *T = dbl ? "double" : "float";
  fma = fma && tab.simple;  // the contracted form exists for packed tables
  std::string body, k = std::string(T) + (tab.simple ? (fma ? ":pf:" : ":p:") : ":g:");
  for (int t = 0; t < tab.nterms; t++) {
    if (tab.simple) {
      const int w = tab.word[t];
      k += std::to_string(w) + ",";
      if (t == 0 || (w & 64))
        body += "    gt_rows<T>(ring, sbytes, S, slot0, thr_off, bx, lane, " +
                std::to_string(w & 7) + ", " + std::to_string(w >> 10) + ", " +
                ((w >> 8) & 1 ? "true" : "false") + ", " + ((w >> 9) & 1 ? "true" : "false") +
                ", row);\n";
      body += "    gt_term<" + std::to_string((w >> 3) & 7) + ", " +
              ((w >> 7) & 1 ? "true" : "false") + ", " + (t == 0 ? "true" : "false") + ", " +
              (fma ? "true" : "false") + ">(row, gt_coef(tab, " + std::to_string(t) +
              ", T()), acc);\n";
    } else {
      const GtFactor &a = tab.a[t], &b = tab.b[t];
      k += std::to_string(a.kind) + "." + std::to_string(a.k) + "." + std::to_string(a.off) + "*" +
           std::to_string(b.kind) + "." + std::to_string(b.k) + "." + std::to_string(b.off) + ",";
      body += "    gt_general_term<T>(" + gt_factor_src(a, "a", t) + ", " +
              gt_factor_src(b, "b", t) + ", " + (t == 0 ? "true" : "false") +
              ", ring, sbytes, S, slot0, thr_off, bx, acc);\n";
    }
  }
  *key = "k_generic_tma:" + k + "vy" + std::to_string(kGtVY) + "pm" +
         std::to_string(PSB_GT_PACKED_MUL);
  std::string src = "#include \"k_generic_tma.cuh\"\nnamespace psb {\nstruct GtCompiledProg {\n"
                    "  static constexpr bool kCompiled = true;\n"
                    "  static constexpr bool kPoints = false;\n  template <typename T>\n"
                    "  static __device__ __forceinline__ void eval(const GtTable &tab, "
                    "const unsigned char *ring, int sbytes, int S, int slot0, int thr_off, "
                    "int bx, int lane, GtBlk<T> &acc) {\n";
  if (tab.simple) src += "    GtRow<T> row[kGtVY];\n";
  else src += "    (void)lane;\n";
  src += body;
  src += "  }\n};\n}  // namespace psb\n";
  src += std::string("extern \"C\" __global__ void __launch_bounds__(psb::kGtThreads, ") +
         (dbl ? "3" : "4") +
         ") psb_generic_tma_compiled(const __grid_constant__ psb::GtMaps maps, "
         "const __grid_constant__ psb::GtTable tab, psb::GridView out, psb::Dom3 d, "
         "const __grid_constant__ psb::GtGeom geo, int *err) {\n  psb::gt_body<" +
         T + ", psb::GtCompiledProg>(maps, tab, out, d, geo, err);\n}\n";
  return src;
}

// The compiled kernel of a table, or nullptr (the interpreting kernel
// runs). Never compiles while the stream is being captured: the first
// iteration of every run is eager, so a captured one finds its kernel cached.
static CUfunction gt_jit(const GtTable &tab, bool dbl, bool fma, cudaStream_t s,
                         size_t smem_optin) {
  if (!generic_compile_on()) return nullptr;
  std::string key;
  const std::string src = gt_jit_source(tab, dbl, fma, &key);
  CUfunction fn = nullptr;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return rtc_cached(key, &fn) == PSB_OK ? fn : nullptr;  // no compile or module load here
  const std::vector<std::string> opts = {"-DPSB_GT_VY=" + std::to_string(kGtVY),
                                         "-DPSB_GT_PACKED_MUL=" + std::to_string(PSB_GT_PACKED_MUL)};
  if (rtc_function(key, src, "psb_generic_tma_compiled", opts, (int)smem_optin, &fn) != PSB_OK)
    return nullptr;
  return fn;
}

// Geometry, tensor maps and grid size of a TMA launch over the staged grids
// of plan p (the map's grids at p.slots), writing `og` over domain d.
template <typename T>
static psb_status gt_geometry(MapImpl &m, const GtPlan &p, GridImpl *og, const Dom3 &d,
                              GtGeom &geo, GtMaps &maps, int64_t *nblocks_out) {
  constexpr int V = 16 / sizeof(T);
  Runtime &r = rt();
  memset(&geo, 0, sizeof(geo));
  geo.tx_threads = 32;
  const int TX = geo.tx_threads * V, TY = (kGtConsumers / geo.tx_threads) * kGtVY;
  geo.bx = TX + 2 * V;
  geo.by = TY + 2 * kGtR;
  geo.ngrids = p.ngrids;
  geo.plane_elems = (geo.bx * geo.by * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
  geo.stage_bytes = geo.ngrids * geo.plane_elems * (int)sizeof(T);
  geo.zmin = p.zmin;
  geo.window = p.zmax - p.zmin + 1;
  geo.stages = geo.window + 2;
  geo.x_base = d.lo[0] / V * V;
  geo.tiles_x = (d.hi[0] - geo.x_base + TX - 1) / TX;
  geo.tiles_y = (d.hi[1] - d.lo[1] + TY - 1) / TY;
  geo.vec_store = tma_eligible(og) ? 1 : 0;
  // z chunks: long enough to amortise the window's extra planes, short
  // enough for a few CTAs per SM.
  const int64_t tiles = (int64_t)geo.tiles_x * geo.tiles_y;
  geo.zchunk = 32;
  while (geo.zchunk > 4 && tiles * ((d.hi[2] - d.lo[2] + geo.zchunk - 1) / geo.zchunk) <
                               (int64_t)r.sm_count * 4)
    geo.zchunk /= 2;
  const int nzc = (d.hi[2] - d.lo[2] + geo.zchunk - 1) / geo.zchunk;
  const int64_t nblocks = tiles * nzc;
  if (nblocks > 0x7fffffff) return PSB_ERR_UNSUPPORTED;
  memset(&maps, 0, sizeof(maps));
  for (int i = 0; i < p.ngrids; i++) {
    GridImpl *g = m.grids[p.slots[i]];
    const CUtensorMap *tm = nullptr;
    if (get_tmap(g, geo.bx, geo.by, &tm) != PSB_OK) return PSB_ERR_UNSUPPORTED;
    maps.m[i] = *tm;
    const bool pitched = g->layout == PSB_LAYOUT_PITCHED;
    geo.ax0[i] = pitched ? g->pad_left : 0;
    geo.ay0[i] = pitched ? g->halo : 0;
    geo.az0[i] = pitched ? g->halo : 0;
  }
  *nblocks_out = nblocks;
  return PSB_OK;
}

template <typename T>
static psb_status gt_launch(MapImpl &m, const psb_generic_stencil &desc, const GtPlan &p,
                            cudaStream_t s, int64_t *launches) {
  Runtime &r = rt();
  GridImpl *og = m.grids[desc.out_grid];
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    d.lo[i] = m.dom.local_min[i];
    d.hi[i] = m.dom.local_max[i];
  }
  GtGeom geo;
  GtMaps maps;
  int64_t nblocks = 0;
  if (gt_geometry<T>(m, p, og, d, geo, maps, &nblocks) != PSB_OK) return PSB_ERR_UNSUPPORTED;
  GtTable tab;
  memset(&tab, 0, sizeof(tab));
  tab.nterms = desc.nterms;
  tab.has_post = desc.has_post;
  for (int t = 0; t < desc.nterms; t++) {
    tab.a[t] = gt_compact(desc.terms[t].a, p, geo.plane_elems, geo.bx);
    tab.b[t] = gt_compact(desc.terms[t].b, p, geo.plane_elems, geo.bx);
  }
  if (desc.has_post) tab.post = gt_compact(desc.post, p, geo.plane_elems, geo.bx);
  // The packed form when every term is one read times a constant.
  tab.simple = !desc.has_post;
  for (int t = 0; t < desc.nterms && tab.simple; t++)
    if ((tab.a[t].kind == 2) == (tab.b[t].kind == 2)) tab.simple = 0;
  if (tab.simple) {
    // Runs of consecutive terms on the same row (plane, grid, dy) share one
    // load; each run records whether it needs the neighbouring lanes.
    int run_start = 0;
    for (int t = 0; t < desc.nterms; t++) {
      const GtFactor &rd = tab.a[t].kind == 2 ? tab.a[t] : tab.b[t];
      const GtFactor &cf = tab.a[t].kind == 2 ? tab.b[t] : tab.a[t];
      const int dx = desc.terms[t].a.grid >= 0 ? desc.terms[t].a.offset[0]
                                               : desc.terms[t].b.offset[0];
      const int rowoff = rd.off - dx;
      const bool fresh = t == 0 || rowoff != (tab.word[t - 1] >> 10) || rd.k != (tab.word[t - 1] & 7);
      if (fresh) run_start = t;
      tab.word[t] = (rowoff << 10) | ((cf.kind == 1) << 7) | (fresh << 6) | ((dx + 2) << 3) | rd.k;
      tab.coef[t] = cf.kind == 1 ? 1.0 : cf.c;
      tab.coef32[t] = (float)tab.coef[t];
      if (dx > 0) tab.word[run_start] |= 1 << 8;
      if (dx < 0) tab.word[run_start] |= 1 << 9;
    }
  }
  const size_t smem = 128 + 512 + (size_t)geo.stages * geo.stage_bytes;
  if (smem > r.smem_optin) return PSB_ERR_UNSUPPORTED;
  static size_t configured[2] = {0, 0};
  size_t &conf = configured[sizeof(T) == 8];
  if (smem > conf) {
    PSB_TRY(cudaFuncSetAttribute(k_generic_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)r.smem_optin));
    PSB_TRY(cudaFuncSetAttribute(k_generic_tma<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    conf = r.smem_optin;
  }
  // Periodic and clamped reads take the halo: refresh it where it is stale.
  for (int i = 0; i < p.ngrids; i++) {
    GridImpl *g = m.grids[p.slots[i]];
    if (p.mode[i] != PSB_BOUNDARY_NONE && g->ghost_valid != p.mode[i])
      PSB_CHECK(launch_halo_fill(g, p.mode[i], s));
  }
  CUfunction fn = gt_jit(tab, sizeof(T) == 8, r.fp_mode == PSB_FP_FMA, s, r.smem_optin);
  GridView ov = og->view();
  if (fn) {
    void *args[] = {&maps, &tab, &ov, &d, &geo, &r.d_error};
    PSB_CHECK(rtc_launch(fn, (unsigned)nblocks, kGtThreads, (unsigned)smem, s, args));
  } else {
    k_generic_tma<T><<<(unsigned)nblocks, kGtThreads, smem, s>>>(maps, tab, ov, d, geo,
                                                                r.d_error);
  }
  (*launches)++;
  g_last_generic_impl = PSB_IMPL_TMA;
  g_last_generic_compiled = fn ? 1 : 0;
  return PSB_OK;
}

// PSB_ERR_UNSUPPORTED when the map does not fit the TMA path (the caller
// then runs k_generic).
psb_status generic_tma_launch(MapImpl &m, const GenericDesc &gd, int color, cudaStream_t s,
                              int64_t *launches) {
  const psb_generic_stencil &desc = gd.host;
  g_last_generic_impl = PSB_IMPL_GENERIC;
  if (desc.ndims != 3 || color >= 0 || desc.nterms < 1) return PSB_ERR_UNSUPPORTED;
  if (desc.accum_type != PS_FLOAT && desc.accum_type != PS_DOUBLE) return PSB_ERR_UNSUPPORTED;
  if (desc.grid_type[desc.out_grid] != desc.accum_type) return PSB_ERR_UNSUPPORTED;
  for (int k = 0; k < 3; k++)
    if (desc.grid_axes[desc.out_grid][k] != k) return PSB_ERR_UNSUPPORTED;
  for (int i = 0; i < 3; i++)
    if (m.dom.local_max[i] <= m.dom.local_min[i]) return PSB_ERR_UNSUPPORTED;
  GtPlan p;
  for (int t = 0; t < desc.nterms; t++)
    if (!gt_factor_ok(desc, m, desc.terms[t].a, p) || !gt_factor_ok(desc, m, desc.terms[t].b, p))
      return PSB_ERR_UNSUPPORTED;
  if (desc.has_post && !gt_factor_ok(desc, m, desc.post, p)) return PSB_ERR_UNSUPPORTED;
  if (p.ngrids == 0) return PSB_ERR_UNSUPPORTED;
  for (int i = 0; i < p.ngrids; i++)
    if (!tma_eligible(m.grids[p.slots[i]])) return PSB_ERR_UNSUPPORTED;
  GridImpl *og = m.grids[desc.out_grid];
  if (og->pub.num_dims != 3 || og->type != desc.accum_type) return PSB_ERR_UNSUPPORTED;
  return desc.accum_type == PS_FLOAT ? gt_launch<float>(m, desc, p, s, launches)
                                     : gt_launch<double>(m, desc, p, s, launches);
}

void generic_note_impl(int impl) { g_last_generic_impl = impl; }

static int g_last_compiled_staged = 0;

template <typename T>
static psb_status staged_run(MapImpl &m, psb_compiled_staged fn, const GtPlan &p, GridImpl *og,
                             const Dom3 &d, GtTable &tab, cudaStream_t s) {
  Runtime &r = rt();
  GtGeom geo;
  GtMaps maps;
  int64_t nblocks = 0;
  if (gt_geometry<T>(m, p, og, d, geo, maps, &nblocks) != PSB_OK) return PSB_ERR_UNSUPPORTED;
  const size_t smem = 128 + 512 + (size_t)geo.stages * geo.stage_bytes;
  if (smem > r.smem_optin) return PSB_ERR_UNSUPPORTED;
  for (int k = 0; k < PSB_MAX_TERMS && k < m.nparams; k++) {
    tab.coef[k] = m.params[k];
    tab.coef32[k] = (float)m.params[k];
  }
  GridView ov = og->view();
  return fn(&maps, &tab, &ov, &d, &geo, r.d_error, (unsigned)nblocks, (unsigned)smem, (void *)s);
}

// A compiled stencil's staged form: the map must read only grids of the
// stencil's type that TMA can stage (at most four distinct ones), never the
// grid it emits into. When every read range stays inside its grid over the
// whole domain the unchecked form runs; when one may leave its grid (reads
// under face tests) the checked form runs, which needs the domain inside
// every grid read (a read at the point's own coordinate on an axis is then
// inside, so only the axes a read leaves the point on are checked).
// Otherwise the function keeps its own form, which checks every read.
psb_status compiled_staged_launch(MapImpl &m, const psb_compiled_stencil &cd, GridImpl **views,
                                  int color, cudaStream_t s) {
  g_last_compiled_staged = 0;
  const Runtime &r = rt();
  if (!cd.staged || r.impl == PSB_IMPL_PLAIN || r.impl == PSB_IMPL_GENERIC)
    return PSB_ERR_UNSUPPORTED;
  if (color >= 0 || cd.ndims != 3 || cd.nviews != cd.ngrids || m.nparams > PSB_MAX_TERMS)
    return PSB_ERR_UNSUPPORTED;
  GridImpl *og = views[cd.staged_emit];
  if (og->type != cd.staged_type || og->pub.num_dims != 3) return PSB_ERR_UNSUPPORTED;
  Dom3 d;
  for (int i = 0; i < 3; i++) {
    d.lo[i] = m.dom.local_min[i];
    d.hi[i] = m.dom.local_max[i];
    if (d.hi[i] <= d.lo[i]) return PSB_ERR_UNSUPPORTED;
  }
  GtPlan p;
  GtTable tab;
  memset(&tab, 0, sizeof(tab));
  bool inside = true, dom_inside = true;
  for (int i = 0; i < cd.ngrids; i++) {
    GridImpl *g = views[i];
    tab.slot_grid[i] = -1;
    for (int k = 0; k < 3; k++) tab.slot_dims[i][k] = g->pub.dim[k];
    if (cd.read_lo[i][0] > cd.read_hi[i][0]) continue;  // not read
    if (g == og || g->type != cd.staged_type || g->pub.num_dims != 3 || !tma_eligible(g))
      return PSB_ERR_UNSUPPORTED;
    // Periodic reads take the wrapped values from the halo of a pitched grid.
    // The read range of such a grid covers its plain reads too, so the range
    // test below stays a sound choice between the two forms (plain reads
    // outside the grid are checked; periodic ones never are).
    const bool per = cd.read_periodic[i] != 0;
    if (per && (g->layout != PSB_LAYOUT_PITCHED || g->halo < kGtR)) return PSB_ERR_UNSUPPORTED;
    for (int k = 0; k < 3; k++) {
      if (d.lo[k] + cd.read_lo[i][k] < 0 || d.hi[k] - 1 + cd.read_hi[i][k] > g->pub.dim[k] - 1)
        inside = false;
      if (d.hi[k] > g->pub.dim[k]) dom_inside = false;
    }
    int gi = -1;
    for (int j = 0; j < p.ngrids; j++)
      if (views[p.slots[j]] == g) gi = j;
    if (gi < 0) {
      if (p.ngrids == kGtMaxGrids) return PSB_ERR_UNSUPPORTED;
      gi = p.ngrids++;
      p.slots[gi] = i;
      p.mode[gi] = PSB_BOUNDARY_NONE;
    }
    if (per) p.mode[gi] = PSB_BOUNDARY_PERIODIC;
    tab.slot_grid[i] = gi;
    p.zmin = std::min(p.zmin, cd.read_lo[i][2]);
    p.zmax = std::max(p.zmax, cd.read_hi[i][2]);
  }
  if (p.ngrids == 0) return PSB_ERR_UNSUPPORTED;
  if (!inside && (!cd.staged_checked || !dom_inside)) return PSB_ERR_UNSUPPORTED;
  // Periodic reads take the halo: refresh it where it is stale.
  for (int i = 0; i < p.ngrids; i++) {
    GridImpl *g = views[p.slots[i]];
    if (p.mode[i] != PSB_BOUNDARY_NONE && g->ghost_valid != p.mode[i])
      PSB_CHECK(launch_halo_fill(g, p.mode[i], s));
  }
  const psb_compiled_staged fn = inside ? cd.staged : cd.staged_checked;
  tab.read_err = r.d_error + 1;  // where the own form reports reads outside a grid
  const psb_status st = cd.staged_type == PS_FLOAT ? staged_run<float>(m, fn, p, og, d, tab, s)
                                                   : staged_run<double>(m, fn, p, og, d, tab, s);
  if (st == PSB_OK) g_last_compiled_staged = inside ? 1 : 2;
  return st;
}

}  // namespace psb

extern "C" psb_status psb_generic_last_impl(int *impl) {
  if (!impl) return psb::set_status(PSB_ERR_INVALID);
  *impl = psb::g_last_generic_impl;
  return PSB_OK;
}

extern "C" psb_status psb_generic_last_compiled(int *compiled) {
  if (!compiled) return psb::set_status(PSB_ERR_INVALID);
  *compiled = psb::g_last_generic_impl == PSB_IMPL_TMA ? psb::g_last_generic_compiled : 0;
  return PSB_OK;
}

extern "C" psb_status psb_compiled_last_staged(int *staged) {
  if (!staged) return psb::set_status(PSB_ERR_INVALID);
  *staged = psb::g_last_compiled_staged;
  return PSB_OK;
}

extern "C" psb_status psb_set_generic_compile(int on) {
  psb::g_generic_compile = on ? 1 : 0;
  return PSB_OK;
}
