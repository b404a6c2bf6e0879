// Serving loop (placeholder until continuous batching lands).
#include "thv_internal.h"

using namespace thv;

extern "C" {
thv_status thv_serve_start(thv_graph *, const thv_serve_opts *, thv_server **) {
  return fail(THV_EUNSUPPORTED, "serving not built yet");
}
thv_status thv_serve_submit(thv_server *, thv_algo, uint32_t, uint64_t *) {
  return fail(THV_EUNSUPPORTED, "serving not built yet");
}
thv_status thv_serve_poll(thv_server *, uint64_t, uint32_t *, thv_query_stats *) {
  return fail(THV_EUNSUPPORTED, "serving not built yet");
}
thv_status thv_serve_wait(thv_server *, uint64_t, uint32_t *, thv_query_stats *, uint32_t) {
  return fail(THV_EUNSUPPORTED, "serving not built yet");
}
thv_status thv_serve_stop(thv_server *) { return THV_OK; }
}
