#include "internal.h"
extern "C" {
psb_status psb_server_create(size_t mem_budget_bytes, int max_slots, int mode, psb_server **s) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_submit(psb_server *s, const psb_request *req, int64_t *id) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_cancel(psb_server *s, int64_t id) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_wait(psb_server *s, int64_t id, float *out, double timeout_s, psb_result *res) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_stats(psb_server *s, int64_t *completed, int64_t *rounds, int64_t *launches, size_t *peak_bytes) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
psb_status psb_server_destroy(psb_server *s) { return psb::set_status(PSB_ERR_UNSUPPORTED); }
}
