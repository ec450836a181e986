// Batched form: placeholder.
#include "engine.h"

extern "C" {
sme_status sme_batch_opts_default(sme_batch_opts* o) {
  if (!o) return SME_ERR_INVALID_ARG;
  *o = sme_batch_opts{};
  o->autotune = 1;
  o->use_graph = 1;
  return SME_OK;
}
sme_status sme_batch_count(sme_graph* const*, const int32_t*, uint64_t, const sme_batch_opts*, uint64_t*) {
  return SME_ERR_INVALID_ARG;
}
sme_status sme_batch_prepare(sme_graph* const*, const int32_t*, uint64_t, const sme_batch_opts*,
                             sme_batch_plan**) {
  return SME_ERR_INVALID_ARG;
}
sme_status sme_batch_run(sme_batch_plan*, uint64_t*, double*) { return SME_ERR_INVALID_ARG; }
sme_status sme_batch_describe(const sme_batch_plan*, int32_t*, int32_t*, uint64_t*) { return SME_ERR_INVALID_ARG; }
sme_status sme_batch_free(sme_batch_plan*) { return SME_OK; }
}
