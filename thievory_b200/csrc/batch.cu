// Batched multi-source BFS / SSSP (placeholder until the 64-wide kernels land).
#include "thv_internal.h"

namespace thv {

struct BatchState {};

thv_status run_batch(thv_graph *g, thv_algo algo, const uint32_t *sources,
                     uint32_t n, const thv_batch_opts *o, uint32_t *out,
                     thv_stats *stats) {
  (void)g; (void)algo; (void)sources; (void)n; (void)o; (void)out; (void)stats;
  return fail(THV_EUNSUPPORTED, "batched runs not built yet");
}

void batch_free(thv_graph *g) {
  delete g->bs;
  g->bs = nullptr;
}

}  // namespace thv
