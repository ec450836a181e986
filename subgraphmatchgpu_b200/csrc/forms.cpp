// Served form: placeholder.
#include "../../include/sme.h"

extern "C" {
sme_status sme_server_opts_default(sme_server_opts* o) {
  if (!o) return SME_ERR_INVALID_ARG;
  *o = sme_server_opts{};
  o->slots = 4;
  o->queue_capacity = 4096;
  return SME_OK;
}
sme_status sme_server_create(const sme_server_opts*, sme_server**) { return SME_ERR_INVALID_ARG; }
sme_status sme_server_add_graph(sme_server*, sme_graph*, int32_t*) { return SME_ERR_INVALID_ARG; }
sme_status sme_server_submit(sme_server*, int32_t, sme_graph*, const sme_opts*, uint64_t*) {
  return SME_ERR_INVALID_ARG;
}
sme_status sme_server_poll(sme_server*, uint64_t, uint64_t*, double*) { return SME_ERR_INVALID_ARG; }
sme_status sme_server_wait(sme_server*, uint64_t, uint64_t*, double*) { return SME_ERR_INVALID_ARG; }
sme_status sme_server_stats(sme_server*, uint64_t*, uint64_t*, uint64_t*) { return SME_ERR_INVALID_ARG; }
sme_status sme_server_destroy(sme_server*) { return SME_OK; }
}
