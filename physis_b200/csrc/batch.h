// Host-side batch member record shared by the batching and serving code.
#pragma once

#include <vector>

#include "internal.h"

namespace psb {

enum { BK_DIFF7 = 0, BK_DIFF7P = 1, BK_HIMENO = 2 };

struct BatchMemberHost {
  int kind = 0;            // 0 diffusion clamped, 1 diffusion periodic, 2 Himeno
  int kernel_id = 0;       // PSB_KERNEL_*
  GridImpl *grids[14] = {};
  int ngrids = 0;
  double params[PSB_MAX_PARAMS] = {};
  int nparams = 0;
  int steps = 0;           // total steps of the solve
  int check_every = 0;     // residual check interval (0: none)
  double tol = 0.0;        // relative residual tolerance (0: run all steps)
  int64_t points = 0;      // lattice updates per step
  int force_tx = 0;        // autotuner trials: consumer threads along x (0: choose)
  int force_zc = 0;        // autotuner trials: planes per item (0: choose)
  int force_td = 0;        // autotuner trials: Himeno sweeps per pass, 1 or 2 (0: choose)
  int cur0 = 0;            // which of grids[0], grids[1] holds the state at the first step
};

}  // namespace psb

struct psb_batch;

namespace psb {
psb_status batch_prepare(psb_batch *b, const std::vector<int> &steps, const std::vector<int> &step0);
psb_status batch_launch_persistent(psb_batch *b, cudaStream_t s, int64_t *launches);
psb_status batch_launch_graph(psb_batch *b, cudaStream_t s, int64_t *launches);
psb_status batch_add_member(psb_batch *b, const BatchMemberHost &m);
psb_status batch_read_state(psb_batch *b, std::vector<int> &stop, std::vector<double> &res);
bool batch_member_wavefront(const psb_batch *b, int i);
// Which of member i's two grids holds its state after `done` local steps of
// the last prepared launch.
int batch_member_cur(const psb_batch *b, int i, int done);
// Server access to a batch's member list (replaced every round).
psb_batch *batch_new();
void batch_set_members(psb_batch *b, const std::vector<BatchMemberHost> &m,
                       const std::vector<double> &res_init);
void batch_delete(psb_batch *b);
}  // namespace psb
