// Serving: continuous batching of stencil solve requests.
//
// A request is one PSStencilRun-style solve (7-point diffusion, clamped or
// periodic, or Himeno Jacobi, float) that runs until its relative residual
// is <= tol at a check or for max_steps steps. A worker thread owns the
// device side:
//
//   admission  -- queued requests are admitted in arrival order while the
//                 bytes of their resident grids fit the memory budget (and a
//                 slot is free); their grids come from a stream-ordered pool,
//                 are filled on the device (copy-in or seeded generation) and
//                 stay resident until the request finishes;
//   rounds     -- admitted requests advance together in one launch of the
//                 persistent batched kernel (one work list over all of them,
//                 each at its own step count); a round takes the requests
//                 with the least remaining work until they fill the GPU at
//                 every step (so small solves finish first rather than all
//                 together), and runs R steps of each, R chosen so a round is
//                 some 20 ms of work; requests admitted while a round runs
//                 join the next one;
//   retirement -- a request that converged (the kernel stops it at the check
//                 step, so no work is spent past it), ran max_steps or was
//                 cancelled leaves the list; its result is copied to the
//                 caller's buffer on a copy stream while the next round runs,
//                 then its grids go back to the pool and its bytes to the
//                 budget.
//
// Each request's arithmetic, check schedule (global step numbers) and
// residual sums (per-tile partials in tile order) are those of running it
// alone, so its result and its stop step do not depend on the mix.
//
// The FIFO mode is the baseline: one request at a time in arrival order,
// each step one launch of the plain (reference-shaped) kernel, residuals by
// a separate pass over the grids at each check.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"

namespace psb {

struct SReq {
  int64_t id = 0;
  psb_request q{};
  int kind = 0;
  size_t bytes = 0;
  double submit_s = 0, start_s = 0, finish_s = 0;
  psb_status status = PSB_OK;
  int steps_done = 0;
  double residual = -1.0;
  std::atomic<bool> cancel{false};
  bool complete = false;
  int skipped = 0;  // consecutive rounds this admitted request was left out of
  int wave_rounds = 0;  // rounds in which its steps overlapped as a wavefront
  int cur = 0;          // which of its two state grids holds the current state
  BatchMemberHost h;
  double res[4] = {0, 0, 0, 0};
  cudaEvent_t copied = nullptr;
  void *stage = nullptr;  // packed result on its way to the host
};

// Lattice updates a round aims at (some 20 ms of device time), and the
// fewest steps a round gives each request.
constexpr double kRoundWork = 1.6e10;
constexpr int kRoundMinSteps = 4;
// A round advances the admitted requests with the least remaining work
// (shortest remaining work first, so small solves finish early instead of
// all finishing together) until their points per step reach kRoundPoints,
// enough tiles to keep every SM busy at every step; a request left out of
// kMaxSkipRounds rounds in a row is always taken.
constexpr int64_t kRoundPoints = 96ll << 20;
constexpr int kMaxSkipRounds = 8;

// Residual terms of two grids (FIFO mode): per-CTA FP64 partials of
// sum (a - b)^2 and sum a^2, combined on the host in CTA order.
constexpr int kNormBlocks = 296;
__global__ void __launch_bounds__(256) k_pair_norm(GridView a, GridView b, double *partials) {
  const int nx = a.n[0], ny = a.n[1], nz = a.n[2];
  const int64_t rows = (int64_t)ny * nz;
  double s0 = 0, s1 = 0;
  for (int64_t r = blockIdx.x * 8 + (threadIdx.x >> 5); r < rows; r += (int64_t)gridDim.x * 8) {
    const int y = (int)(r % ny), z = (int)(r / ny);
    const float *pa = (const float *)a.origin + y * a.sy + z * a.sz;
    const float *pb = (const float *)b.origin + y * b.sy + z * b.sz;
    for (int x = threadIdx.x & 31; x < nx; x += 32) {
      const double u = pa[x], d = u - (double)pb[x];
      s0 += d * d;
      s1 += u * u;
    }
  }
  __shared__ double sh[2][8];
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_down_sync(0xffffffffu, s0, o);
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = s0;
    sh[1][threadIdx.x >> 5] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0, t1 = 0;
    for (int w = 0; w < 8; w++) {
      t0 += sh[0][w];
      t1 += sh[1][w];
    }
    partials[2 * blockIdx.x] = t0;
    partials[2 * blockIdx.x + 1] = t1;
  }
}

}  // namespace psb

using namespace psb;

struct psb_server {
  size_t budget = 0;
  int max_slots = 0;
  int mode = 0;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<SReq *> queue;
  std::unordered_map<int64_t, SReq *> reqs;  // every request not yet returned by wait
  std::deque<int64_t> done_order;            // completed, in completion order
  int64_t next_id = 1;
  bool shutdown = false;
  size_t used = 0, peak = 0;
  int64_t completed = 0, rounds = 0, launches = 0;
  double device_ms = 0;
  // Worker-owned.
  std::vector<SReq *> active;
  std::vector<SReq *> retiring;  // result copy in flight
  psb_batch *batch = nullptr;
  cudaMemPool_t pool = nullptr;
  cudaStream_t copy = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_prev = nullptr;  // end of the previous batched round (trace only)
  bool have_prev = false;
  double create_s = 0;
  double *d_norm = nullptr;
  std::thread worker;
};

namespace psb {

static int request_kind(int kernel_id) {
  switch (kernel_id) {
    case PSB_KERNEL_DIFFUSION7: return BK_DIFF7;
    case PSB_KERNEL_DIFFUSION7_PERIODIC: return BK_DIFF7P;
    case PSB_KERNEL_HIMENO19: return BK_HIMENO;
    default: return -1;
  }
}

static int request_ngrids(int kind) { return kind == BK_HIMENO ? 14 : 2; }

static psb_status request_check(const psb_request *q, size_t *bytes) {
  const int kind = request_kind(q->kernel_id);
  if (kind < 0) return PSB_ERR_UNSUPPORTED;
  if (q->max_steps < 1 || q->tol < 0 || q->check_every < 0 || (q->tol > 0 && q->check_every < 1))
    return PSB_ERR_INVALID;
  if (q->nparams != (kind == BK_HIMENO ? 1 : 7)) return PSB_ERR_INVALID;
  const int lo = kind == BK_HIMENO ? 3 : 4;
  for (int k = 0; k < 3; k++)
    if (q->dims[k] < lo) return PSB_ERR_INVALID;
  *bytes = grid_pitched_bytes(4, q->dims) * request_ngrids(kind);
  return PSB_OK;
}

// Complete a request (server lock held).
static void complete_locked(psb_server *S, SReq *q, psb_status st) {
  q->status = st;
  q->finish_s = now_s();
  q->complete = true;
  S->completed++;
  S->done_order.push_back(q->id);
  S->cv_done.notify_all();
}

static void free_grids(psb_server *S, SReq *q, cudaStream_t s) {
  for (int i = 0; i < q->h.ngrids; i++) grid_free_pool(q->h.grids[i], s);
  q->h.ngrids = 0;
}

// Allocate and fill the grids of an admitted request on the runtime stream.
static psb_status admit_request(psb_server *S, SReq *q) {
  Runtime &r = rt();
  BatchMemberHost &h = q->h;
  h.kind = q->kind;
  h.kernel_id = q->q.kernel_id;
  h.ngrids = 0;
  const int ng = request_ngrids(q->kind);
  for (int i = 0; i < ng; i++) {
    GridImpl *g = nullptr;
    PSB_CHECK(grid_alloc_pool(PS_FLOAT, q->q.dims, S->pool, r.stream, &g));
    h.grids[h.ngrids++] = g;
  }
  const size_t n = (size_t)q->q.dims[0] * q->q.dims[1] * q->q.dims[2];
  if (q->q.init) {
    PSB_CHECK(grid_copy_in_on(h.grids[0], q->q.init, r.stream));
  } else if (q->kind == BK_HIMENO) {
    PSB_CHECK(psb_grid_fill(&h.grids[0]->pub, 3, 0, 0.0, 0.0));
  } else {
    PSB_CHECK(psb_grid_fill(&h.grids[0]->pub, 0, q->q.seed, 0.0, 1.0));
  }
  if (q->kind == BK_HIMENO) {
    // The output p keeps the input's boundary values (the sweep writes the
    // interior only).
    if (q->q.init)
      PSB_CHECK(grid_copy_in_on(h.grids[1], q->q.init, r.stream));
    else
      PSB_CHECK(psb_grid_fill(&h.grids[1]->pub, 3, 0, 0.0, 0.0));
    static const double lo[10] = {0.9, 0.9, 0.9, 0.95 / 6, -0.01, -0.01, -0.01, 0.9, 0.9, 0.9};
    static const double hi[10] = {1.1, 1.1, 1.1, 1.05 / 6, 0.01, 0.01, 0.01, 1.1, 1.1, 1.1};
    for (int k = 0; k < 12; k++) {
      GridImpl *g = h.grids[2 + k];
      if (q->q.coef) {
        PSB_CHECK(grid_copy_in_on(g, q->q.coef + (size_t)k * n, r.stream));
      } else if (k < 10) {
        PSB_CHECK(psb_grid_fill(&g->pub, 0, q->q.seed * 16 + 1 + k, lo[k], hi[k]));
      } else if (k == 10) {
        PSB_CHECK(psb_grid_fill(&g->pub, 2, 0, 0.0, 0.0));
      }  // wrk1 stays zero
    }
  }
  if (q->kind == BK_DIFF7P) {
    PSB_CHECK(launch_halo_fill(h.grids[0], PSB_BOUNDARY_PERIODIC, r.stream));
    h.grids[0]->ghost_valid = PSB_BOUNDARY_PERIODIC;
  }
  for (int i = 0; i < q->q.nparams; i++) h.params[i] = q->q.params[i];
  h.nparams = q->q.nparams;
  h.steps = q->q.max_steps;
  h.check_every = q->q.check_every;
  h.tol = q->q.tol;
  const int *d = q->q.dims;
  h.points = q->kind == BK_HIMENO ? (int64_t)(d[0] - 2) * (d[1] - 2) * (d[2] - 2)
                                  : (int64_t)d[0] * d[1] * d[2];
  q->start_s = now_s();
  return PSB_OK;
}

// Retiring a finished request takes two steps. First, on the runtime stream
// before the next round is launched, its result grid is packed into a dense
// staging buffer (a short HBM pass; once the round's persistent kernel holds
// every SM nothing else would run). Then the copy stream, ordered after the
// pack, moves the dense block to the caller's buffer and releases the
// staging buffer and the grids, while the round runs.
static psb_status retire_pack(psb_server *S, SReq *q) {
  Runtime &r = rt();
  q->stage = nullptr;
  if (q->status == PSB_OK && q->q.out && q->h.ngrids)
    PSB_CHECK(pitched_stage_out(q->h.grids[q->cur], &q->stage, r.stream));
  if (!q->copied) PSB_TRY(cudaEventCreateWithFlags(&q->copied, cudaEventDisableTiming));
  PSB_TRY(cudaEventRecord(q->copied, r.stream));
  return PSB_OK;
}

static psb_status retire_copy(psb_server *S, SReq *q) {
  PSB_TRY(cudaStreamWaitEvent(S->copy, q->copied, 0));
  if (q->stage) {
    const size_t bytes = (size_t)q->q.dims[0] * q->q.dims[1] * q->q.dims[2] * sizeof(float);
    PSB_TRY(cudaMemcpyAsync(q->q.out, q->stage, bytes, cudaMemcpyDeviceToHost, S->copy));
    PSB_TRY(cudaFreeAsync(q->stage, S->copy));
    q->stage = nullptr;
  }
  free_grids(S, q, S->copy);
  PSB_TRY(cudaEventRecord(q->copied, S->copy));
  std::lock_guard<std::mutex> lk(S->mu);
  S->retiring.push_back(q);
  return PSB_OK;
}

static psb_status retire_request(psb_server *S, SReq *q) {
  PSB_CHECK(retire_pack(S, q));
  return retire_copy(S, q);
}

// Complete the retiring requests whose copies are done (server lock held).
static void poll_retiring_locked(psb_server *S, bool wait_all) {
  for (size_t i = 0; i < S->retiring.size();) {
    SReq *q = S->retiring[i];
    cudaError_t e = wait_all ? cudaEventSynchronize(q->copied) : cudaEventQuery(q->copied);
    if (e == cudaErrorNotReady) {
      i++;
      continue;
    }
    if (e != cudaSuccess && q->status == PSB_OK) q->status = cuda_status(e, "result copy");
    S->used -= q->bytes;
    complete_locked(S, q, q->status);
    S->retiring.erase(S->retiring.begin() + i);
  }
}

static double residual_of(const double *r4) {
  if (r4[3] <= 0) return -1.0;
  return r4[1] > 0 ? sqrt(r4[0] / r4[1]) : 0.0;
}

// Take the oldest queued request if it fits the budget and the slot limit
// (server lock held); nullptr if none does.
static SReq *take_one_locked(psb_server *S, size_t pending) {
  if (S->queue.empty()) return nullptr;
  SReq *q = S->queue.front();
  if (S->max_slots > 0 && S->active.size() + pending >= (size_t)S->max_slots) return nullptr;
  if (S->used + q->bytes > S->budget) return nullptr;
  S->queue.pop_front();
  S->used += q->bytes;
  S->peak = std::max(S->peak, S->used);
  return q;
}

// Allocate and fill one taken request (runtime lock held) and add it to the
// active list; a request that cannot be set up completes with its error.
static void admit_one(psb_server *S, SReq *q) {
  const double ta = now_s();
  psb_status st = admit_request(S, q);
  if (__ps_trace)
    fprintf(__ps_trace, "physis_b200 serve: t=%.3f s set up request %lld (kind %d, %dx%dx%d, %.1f MB) "
            "in %.3f ms\n", ta - S->create_s, (long long)q->id, q->kind, q->q.dims[0],
            q->q.dims[1], q->q.dims[2], q->bytes / 1e6, (now_s() - ta) * 1e3);
  if (st != PSB_OK) {
    free_grids(S, q, rt().stream);
    std::lock_guard<std::mutex> lk(S->mu);
    S->used -= q->bytes;
    complete_locked(S, q, st);
    return;
  }
  S->active.push_back(q);
}

static void admit_all(psb_server *S, std::vector<SReq *> &admit) {
  const double ta = now_s();
  for (SReq *q : admit) admit_one(S, q);
  if (__ps_trace && !admit.empty())
    fprintf(__ps_trace, "physis_b200 serve: t=%.3f s admitted %d requests in %.3f ms\n",
            ta - S->create_s, (int)admit.size(), (now_s() - ta) * 1e3);
  admit.clear();
}

// One round of the persistent batched kernel over every active request.
static psb_status run_round(psb_server *S, std::vector<SReq *> &finished) {
  Runtime &r = rt();
  // This round's requests: cancelled ones (to retire them), those waiting
  // too long, then the least remaining work first up to kRoundPoints.
  std::vector<SReq *> order(S->active);
  auto remaining = [](const SReq *q) {
    return (double)q->h.points * (q->q.max_steps - q->steps_done);
  };
  std::stable_sort(order.begin(), order.end(), [&](const SReq *x, const SReq *y) {
    const int px = x->cancel ? 0 : x->skipped >= kMaxSkipRounds ? 1 : 2;
    const int py = y->cancel ? 0 : y->skipped >= kMaxSkipRounds ? 1 : 2;
    if (px != py) return px < py;
    return remaining(x) < remaining(y);
  });
  std::vector<SReq *> round_reqs;
  int64_t points = 0;
  for (SReq *q : order) {
    if (q->cancel || q->skipped >= kMaxSkipRounds || points < kRoundPoints) {
      round_reqs.push_back(q);
      points += q->cancel ? 0 : q->h.points;
      q->skipped = 0;
    } else {
      q->skipped++;
    }
  }
  const int n = (int)round_reqs.size();
  std::vector<BatchMemberHost> hm(n);
  std::vector<int> steps(n), step0(n);
  std::vector<double> res_init(4 * n);
  const int R = (int)std::max<double>(
      kRoundMinSteps, std::min<double>(1000.0, kRoundWork / std::max<int64_t>(1, points)));
  for (int i = 0; i < n; i++) {
    SReq *q = round_reqs[i];
    hm[i] = q->h;
    hm[i].cur0 = q->cur;
    step0[i] = q->steps_done;
    steps[i] = q->cancel ? 0 : std::min(q->q.max_steps - q->steps_done, R);
    for (int k = 0; k < 4; k++) res_init[4 * i + k] = q->res[k];
  }
  const double t0 = now_s();
  batch_set_members(S->batch, hm, res_init);
  PSB_CHECK(batch_prepare(S->batch, steps, step0));
  for (int i = 0; i < n; i++)
    if (batch_member_wavefront(S->batch, i)) round_reqs[i]->wave_rounds++;
  const double t1 = now_s();
  // Results of the previous round: packed now, copied out while this round runs.
  const int nretire = (int)finished.size();
  for (SReq *q : finished) PSB_CHECK(retire_pack(S, q));
  PSB_TRY(cudaEventRecord(S->ev0, r.stream));
  int64_t launches = 0;
  PSB_CHECK(batch_launch_persistent(S->batch, r.stream, &launches));
  PSB_TRY(cudaEventRecord(S->ev1, r.stream));
  for (SReq *q : finished) PSB_CHECK(retire_copy(S, q));
  finished.clear();
  // Requests that arrived meanwhile are set up while the round runs (their
  // allocations and fills queue behind it) and join the next round. Setting
  // one up can take milliseconds of host time (a growing pool maps new
  // memory), so after the first one the worker stops when the round ends
  // and leaves the rest for the next round: the device never waits on a
  // long admission.
  {
    const double ta = now_s();
    int admitted = 0;
    for (;;) {
      if (admitted && cudaEventQuery(S->ev1) != cudaErrorNotReady) break;
      SReq *q;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        q = take_one_locked(S, 0);
      }
      if (!q) break;
      admit_one(S, q);
      admitted++;
    }
    if (__ps_trace && admitted)
      fprintf(__ps_trace, "physis_b200 serve: t=%.3f s admitted %d requests in %.3f ms\n",
              ta - S->create_s, admitted, (now_s() - ta) * 1e3);
  }
  const double t2 = now_s();
  PSB_TRY(cudaEventSynchronize(S->ev1));
  const double t3 = now_s();
  float ms = 0;
  cudaEventElapsedTime(&ms, S->ev0, S->ev1);
  if (__ps_trace) {
    // Device idle time between the previous round's end and this one's start.
    float idle = -1;
    if (S->have_prev) cudaEventElapsedTime(&idle, S->ev_prev, S->ev0);
    fprintf(__ps_trace,
            "physis_b200 serve: t=%.3f s round of %d requests (%lld points/step, %d steps), "
            "%d retired; host prepare %.3f ms, launch+retire %.3f ms, wait %.3f ms; device %.3f "
            "ms, idle before %.3f ms\n",
            t0 - S->create_s, n, (long long)points, R, nretire, (t1 - t0) * 1e3,
            (t2 - t1) * 1e3, (t3 - t2) * 1e3, ms, idle);
    std::swap(S->ev1, S->ev_prev);
    S->have_prev = true;
  }
  int err = 0;
  PSB_TRY(cudaMemcpy(&err, r.d_error, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(r.d_error, 0, sizeof(int));
    return PSB_ERR_TIMEOUT;
  }
  std::vector<int> stop;
  std::vector<double> res;
  PSB_CHECK(batch_read_state(S->batch, stop, res));
  // Periodic writers keep the halo of their outputs current.
  for (int i = 0; i < n; i++) {
    SReq *q = round_reqs[i];
    const int done = stop[i] >= 0 ? stop[i] : steps[i];
    q->cur = batch_member_cur(S->batch, i, done);
    q->steps_done += done;
    for (int k = 0; k < 4; k++) q->res[k] = res[4 * i + k];
    q->residual = residual_of(q->res);
    if (q->kind == BK_DIFF7P)
      for (int k = 0; k < 2; k++) q->h.grids[k]->ghost_valid = PSB_BOUNDARY_PERIODIC;
  }
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->rounds++;
    S->launches += launches;
    S->device_ms += ms;
  }
  std::vector<SReq *> keep;
  std::vector<char> ran(S->active.size(), 0);
  for (int i = 0; i < n; i++) {
    SReq *q = round_reqs[i];
    if (q->cancel) {
      q->status = PSB_ERR_CANCELLED;
      finished.push_back(q);
    } else if (stop[i] >= 0 || q->steps_done >= q->q.max_steps) {
      finished.push_back(q);
    } else {
      continue;
    }
    ran[std::find(S->active.begin(), S->active.end(), q) - S->active.begin()] = 1;
  }
  for (size_t i = 0; i < S->active.size(); i++)
    if (!ran[i]) keep.push_back(S->active[i]);
  S->active.swap(keep);
  return PSB_OK;
}

static void fail_active(psb_server *S, std::vector<SReq *> &finished, psb_status st) {
  Runtime &r = rt();
  cudaStreamSynchronize(r.stream);
  for (SReq *q : S->active) finished.push_back(q);
  S->active.clear();
  for (SReq *q : finished) {
    if (q->status == PSB_OK) q->status = st;
    if (q->stage) cudaFreeAsync(q->stage, r.stream);
    q->stage = nullptr;
    free_grids(S, q, r.stream);
    std::lock_guard<std::mutex> lk(S->mu);
    S->used -= q->bytes;
    complete_locked(S, q, q->status);
  }
  finished.clear();
}

static void worker_batched(psb_server *S) {
  Runtime &r = rt();
  cudaSetDevice(S->device);
  std::vector<SReq *> finished;  // retired after the next round is launched
  for (;;) {
    std::vector<SReq *> admit;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      poll_retiring_locked(S, false);
      // With requests active, new ones are set up while a round runs; with
      // none, one is set up here to start the next round.
      if (S->active.empty())
        if (SReq *q = take_one_locked(S, 0)) admit.push_back(q);
      if (admit.empty() && S->active.empty()) {
        if (!finished.empty()) {
          // Nothing to overlap with: send the results now.
          lk.unlock();
          std::lock_guard<std::recursive_mutex> g(r.mu);
          for (SReq *q : finished)
            if (retire_request(S, q) != PSB_OK) q->status = PSB_ERR_CUDA;
          finished.clear();
          continue;
        }
        if (S->retiring.empty() && S->queue.empty() && S->shutdown) break;
        if (S->retiring.empty())
          S->cv_work.wait_for(lk, std::chrono::milliseconds(50));
        else
          S->cv_work.wait_for(lk, std::chrono::microseconds(200));
        continue;
      }
    }
    std::lock_guard<std::recursive_mutex> g(r.mu);
    admit_all(S, admit);
    if (S->active.empty()) continue;
    psb_status st = run_round(S, finished);
    if (st != PSB_OK) fail_active(S, finished, st);
  }
}

// FIFO baseline: one request alone, one plain-kernel launch per step.
static psb_status run_alone_plain(psb_server *S, SReq *q) {
  Runtime &r = rt();
  BatchMemberHost &h = q->h;
  const int *d = q->q.dims;
  __PSDomain dom = q->kind == BK_HIMENO ? PSDomain3DNew(1, d[0] - 1, 1, d[1] - 1, 1, d[2] - 1)
                                        : PSDomain3DNew(0, d[0], 0, d[1], 0, d[2]);
  __PSGrid *fw[14], *bw[14];
  for (int i = 0; i < h.ngrids; i++) fw[i] = bw[i] = &h.grids[i]->pub;
  bw[0] = &h.grids[1]->pub;
  bw[1] = &h.grids[0]->pub;
  PSStencil ms[2] = {0, 0};
  psb_status st = psb_stencil_map(h.kernel_id, &dom, fw, h.ngrids, h.params, h.nparams, &ms[0]);
  if (st == PSB_OK) st = psb_stencil_map(h.kernel_id, &dom, bw, h.ngrids, h.params, h.nparams, &ms[1]);
  const bool checks = q->q.check_every > 0;
  if (st == PSB_OK && checks && q->kind == BK_HIMENO) {
    st = psb_himeno_residual_enable(ms[0], 1);
    if (st == PSB_OK) st = psb_himeno_residual_enable(ms[1], 1);
  }
  const int ce = q->q.check_every;
  const double tol2 = q->q.tol * q->q.tol;
  double gosa0 = 0;
  int64_t launches = 0;
  PSB_TRY(cudaEventRecord(S->ev0, r.stream));
  while (st == PSB_OK && q->steps_done < q->q.max_steps && !q->cancel) {
    // Run to the next check step (or the end).
    int next = q->q.max_steps;
    if (checks) {
      int c = (q->steps_done / ce + 1) * ce;
      if (q->kind == BK_HIMENO && q->steps_done == 0) c = 1;
      next = std::min(next, c);
    }
    for (int s = q->steps_done; s < next && st == PSB_OK; s++) {
      st = psb_stencil_run(&ms[s & 1], 1, 1);
      launches++;
    }
    if (st != PSB_OK) break;
    q->steps_done = next;
    const bool at_check = checks && (next % ce == 0 || (q->kind == BK_HIMENO && next == 1));
    if (!at_check) continue;
    double a = 0, b = 0;
    if (q->kind == BK_HIMENO) {
      st = psb_himeno_residual(ms[(next - 1) & 1], &a);
      if (st != PSB_OK) break;
      if (next == 1) gosa0 = a;
      b = gosa0;
      q->res[2] = gosa0;
    } else {
      GridView nu = h.grids[next & 1]->view(), old = h.grids[(next - 1) & 1]->view();
      k_pair_norm<<<kNormBlocks, 256, 0, r.stream>>>(nu, old, S->d_norm);
      launches++;
      double part[2 * kNormBlocks];
      cudaError_t e = cudaMemcpyAsync(part, S->d_norm, sizeof(part), cudaMemcpyDeviceToHost, r.stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(r.stream);
      if (e != cudaSuccess) {
        st = cuda_status(e, "residual");
        break;
      }
      for (int i = 0; i < kNormBlocks; i++) {
        a += part[2 * i];
        b += part[2 * i + 1];
      }
    }
    q->res[0] = a;
    q->res[1] = b;
    q->res[3] = next;
    q->residual = residual_of(q->res);
    if (tol2 > 0 && a <= tol2 * b) break;
  }
  cudaEventRecord(S->ev1, r.stream);
  cudaEventSynchronize(S->ev1);
  float ms_ = 0;
  cudaEventElapsedTime(&ms_, S->ev0, S->ev1);
  for (int i = 0; i < 2; i++)
    if (ms[i]) psb_stencil_free(ms[i]);
  if (q->cancel && st == PSB_OK) st = PSB_ERR_CANCELLED;
  q->cur = q->steps_done & 1;  // this loop alternates the two maps step by step
  std::lock_guard<std::mutex> lk(S->mu);
  S->rounds++;
  S->launches += launches;
  S->device_ms += ms_;
  return st;
}

static void worker_fifo(psb_server *S) {
  Runtime &r = rt();
  cudaSetDevice(S->device);
  for (;;) {
    SReq *q = nullptr;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      poll_retiring_locked(S, false);
      if (S->queue.empty()) {
        if (S->shutdown && S->retiring.empty()) break;
        S->cv_work.wait_for(lk, S->retiring.empty() ? std::chrono::microseconds(50000)
                                                    : std::chrono::microseconds(200));
        continue;
      }
      q = S->queue.front();
      S->queue.pop_front();
      S->used += q->bytes;
      S->peak = std::max(S->peak, S->used);
    }
    std::lock_guard<std::recursive_mutex> g(r.mu);
    const int old_impl = r.impl;
    const bool old_graph = r.use_graph;
    r.impl = PSB_IMPL_PLAIN;
    r.use_graph = false;
    psb_status st = admit_request(S, q);
    if (st == PSB_OK) st = run_alone_plain(S, q);
    r.impl = old_impl;
    r.use_graph = old_graph;
    q->status = st;
    if (st == PSB_OK || st == PSB_ERR_CANCELLED) {
      if (retire_request(S, q) == PSB_OK) continue;
      q->status = PSB_ERR_CUDA;
    }
    cudaStreamSynchronize(r.stream);
    free_grids(S, q, r.stream);
    std::lock_guard<std::mutex> lk(S->mu);
    S->used -= q->bytes;
    complete_locked(S, q, q->status);
  }
}

}  // namespace psb

extern "C" {

psb_status psb_server_request_bytes(const psb_request *req, size_t *bytes) {
  if (!req || !bytes) return set_status(PSB_ERR_INVALID);
  psb_status st = request_check(req, bytes);
  return st == PSB_OK ? PSB_OK : set_status(st);
}

psb_status psb_server_create(size_t mem_budget_bytes, int max_slots, int mode, psb_server **out) {
  if (!out || max_slots < 0 || (mode != PSB_SERVE_BATCHED && mode != PSB_SERVE_FIFO))
    return set_status(PSB_ERR_INVALID);
  *out = nullptr;
  PSB_CHECK(ensure_init());
  Runtime &r = rt();
  psb_server *S = new psb_server();
  S->budget = mem_budget_bytes;
  S->max_slots = max_slots;
  S->mode = mode;
  S->device = r.device;
  S->create_s = now_s();
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = r.device;
  cudaError_t e = cudaMemPoolCreate(&S->pool, &props);
  if (e == cudaSuccess) {
    // Keep freed blocks in the pool: the budget, not the driver, bounds it.
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->copy, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&S->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&S->ev1);
  if (e == cudaSuccess) e = cudaEventCreate(&S->ev_prev);
  if (e == cudaSuccess) e = cudaMalloc(&S->d_norm, sizeof(double) * 2 * kNormBlocks);
  if (e != cudaSuccess) {
    psb_status st = cuda_status(e, "psb_server_create");
    if (S->pool) cudaMemPoolDestroy(S->pool);
    if (S->copy) cudaStreamDestroy(S->copy);
    if (S->ev0) cudaEventDestroy(S->ev0);
    if (S->ev1) cudaEventDestroy(S->ev1);
    if (S->ev_prev) cudaEventDestroy(S->ev_prev);
    delete S;
    return st;
  }
  S->batch = batch_new();
  S->worker = std::thread(mode == PSB_SERVE_BATCHED ? worker_batched : worker_fifo, S);
  *out = S;
  return PSB_OK;
}

psb_status psb_server_submit(psb_server *S, const psb_request *req, int64_t *id) {
  if (!S || !req) return set_status(PSB_ERR_INVALID);
  size_t bytes = 0;
  psb_status st = request_check(req, &bytes);
  if (st != PSB_OK) return set_status(st);
  if (bytes > S->budget) return set_status(PSB_ERR_NOMEM);
  SReq *q = new SReq();
  q->q = *req;
  q->kind = request_kind(req->kernel_id);
  q->bytes = bytes;
  q->submit_s = now_s();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->shutdown) {
      delete q;
      return set_status(PSB_ERR_INVALID);
    }
    q->id = S->next_id++;
    S->reqs[q->id] = q;
    S->queue.push_back(q);
  }
  S->cv_work.notify_one();
  if (id) *id = q->id;
  return PSB_OK;
}

psb_status psb_server_cancel(psb_server *S, int64_t id) {
  if (!S) return set_status(PSB_ERR_INVALID);
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return set_status(PSB_ERR_INVALID);
  SReq *q = it->second;
  if (q->complete) return PSB_OK;
  auto qi = std::find(S->queue.begin(), S->queue.end(), q);
  if (qi != S->queue.end()) {
    S->queue.erase(qi);
    complete_locked(S, q, PSB_ERR_CANCELLED);
    return PSB_OK;
  }
  q->cancel = true;
  return PSB_OK;
}

psb_status psb_server_wait(psb_server *S, int64_t id, double timeout_s, psb_result *res) {
  if (!S) return set_status(PSB_ERR_INVALID);
  std::unique_lock<std::mutex> lk(S->mu);
  const auto deadline =
      std::chrono::steady_clock::now() +
      std::chrono::duration_cast<std::chrono::steady_clock::duration>(
          std::chrono::duration<double>(timeout_s < 0 ? 0 : timeout_s));
  for (;;) {
    SReq *q = nullptr;
    if (id >= 0) {
      auto it = S->reqs.find(id);
      if (it == S->reqs.end()) return set_status(PSB_ERR_INVALID);
      if (it->second->complete) q = it->second;
    } else {
      while (!S->done_order.empty() && !S->reqs.count(S->done_order.front()))
        S->done_order.pop_front();
      if (!S->done_order.empty()) q = S->reqs[S->done_order.front()];
      else if (S->reqs.empty()) return set_status(PSB_ERR_INVALID);
    }
    if (q) {
      if (res) {
        res->id = q->id;
        res->status = q->status;
        res->steps_done = q->steps_done;
        res->residual = q->residual;
        res->wave_rounds = q->wave_rounds;
        res->submit_s = q->submit_s;
        res->start_s = q->start_s;
        res->finish_s = q->finish_s;
      }
      S->reqs.erase(q->id);
      if (q->copied) cudaEventDestroy(q->copied);
      delete q;
      return PSB_OK;
    }
    if (timeout_s < 0) {
      S->cv_done.wait(lk);
    } else if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
      return set_status(PSB_ERR_TIMEOUT);
    }
  }
}

psb_status psb_server_stats(psb_server *S, int64_t *completed, int64_t *rounds,
                            int64_t *launches, size_t *peak_bytes, double *device_ms) {
  if (!S) return set_status(PSB_ERR_INVALID);
  std::lock_guard<std::mutex> lk(S->mu);
  if (completed) *completed = S->completed;
  if (rounds) *rounds = S->rounds;
  if (launches) *launches = S->launches;
  if (peak_bytes) *peak_bytes = S->peak;
  if (device_ms) *device_ms = S->device_ms;
  return PSB_OK;
}

psb_status psb_server_destroy(psb_server *S) {
  if (!S) return set_status(PSB_ERR_INVALID);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->shutdown = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  cudaStreamSynchronize(S->copy);
  cudaStreamSynchronize(rt().stream);
  for (auto &kv : S->reqs) {
    if (kv.second->copied) cudaEventDestroy(kv.second->copied);
    delete kv.second;
  }
  batch_delete(S->batch);
  cudaFree(S->d_norm);
  cudaEventDestroy(S->ev0);
  cudaEventDestroy(S->ev1);
  cudaEventDestroy(S->ev_prev);
  cudaStreamDestroy(S->copy);
  cudaMemPoolDestroy(S->pool);
  delete S;
  return PSB_OK;
}

}  // extern "C"
