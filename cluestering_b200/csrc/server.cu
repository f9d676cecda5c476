// server.cu — serving loop (continuous batching). Filled in below the first
// correct clustering path.
#include "abi_internal.h"

using namespace clue_impl;

extern "C" {
clue_status clue_server_create(clue_server**, const clue_server_config*, const clue_params*) {
  return fail(CLUE_ERR_RUNTIME, "serving is not available in this build");
}
clue_status clue_server_submit(clue_server*, const clue_points*, uint64_t*) {
  return fail(CLUE_ERR_RUNTIME, "serving is not available in this build");
}
clue_status clue_server_poll(clue_server*, uint64_t) {
  return fail(CLUE_ERR_RUNTIME, "serving is not available in this build");
}
clue_status clue_server_drain(clue_server*) {
  return fail(CLUE_ERR_RUNTIME, "serving is not available in this build");
}
clue_status clue_server_stats_get(clue_server*, clue_server_stats*) {
  return fail(CLUE_ERR_RUNTIME, "serving is not available in this build");
}
clue_status clue_server_latencies(clue_server*, double*, int64_t, int64_t*) {
  return fail(CLUE_ERR_RUNTIME, "serving is not available in this build");
}
clue_status clue_server_destroy(clue_server*) { return CLUE_OK; }
}
