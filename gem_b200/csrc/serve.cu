// Serving entry points: continuous batching with memory-based admission.
#include <cstring>
#include <deque>
#include <map>

#include "ctx.h"

extern "C" gem_status gem_submit(gem_ctx *ctx, const gem_query *q, int mode, uint64_t *ticket) {
  (void)ctx; (void)q; (void)mode; (void)ticket;
  return GEM_ERR_STATE;
}

extern "C" gem_status gem_poll(gem_ctx *ctx, uint64_t ticket, gem_result *res, int *done) {
  (void)ctx; (void)ticket; (void)res; (void)done;
  return GEM_ERR_STATE;
}
