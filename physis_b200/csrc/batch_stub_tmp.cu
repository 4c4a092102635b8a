#include "internal.h"
extern "C" {
psb_status psb_batch_create(psb_batch **b) { (void)b; return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_batch_add(psb_batch *b, int kernel_id, __PSGrid *const *grids, int ngrids,
                         const double *params, int nparams, int steps, int *member) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_batch_run(psb_batch *b, int mode) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_batch_stats(psb_batch *b, double *device_ms, int64_t *launches, int64_t *lattice_updates) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_batch_free(psb_batch *b) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_create(size_t mem_budget_bytes, int max_slots, int mode, psb_server **s) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_submit(psb_server *s, const psb_request *req, int64_t *id) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_cancel(psb_server *s, int64_t id) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_wait(psb_server *s, int64_t id, float *out, double timeout_s, psb_result *res) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_stats(psb_server *s, int64_t *completed, int64_t *rounds, int64_t *launches, size_t *peak_bytes) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_destroy(psb_server *s) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
}
