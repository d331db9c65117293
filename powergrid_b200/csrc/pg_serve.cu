// Request server: placeholder until the continuous-batching loop lands.
#include "pg_ops.cuh"

using namespace pg;

extern "C" {
pg_status pg_server_create(pg_server* out, const pg_server_config*) {
  if (out) *out = nullptr;
  return set_error(PG_INVALID_ARG, "server not built yet");
}
pg_status pg_server_destroy(pg_server) { return PG_OK; }
pg_status pg_submit(pg_server, const pg_request*, uint64_t*) { return set_error(PG_INVALID_ARG, "server not built yet"); }
pg_status pg_poll(pg_server, uint64_t, pg_request_stats*) { return set_error(PG_INVALID_ARG, "server not built yet"); }
pg_status pg_wait(pg_server, uint64_t, pg_request_stats*) { return set_error(PG_INVALID_ARG, "server not built yet"); }
pg_status pg_cancel(pg_server, uint64_t) { return set_error(PG_INVALID_ARG, "server not built yet"); }
uint64_t pg_request_footprint(const pg_request*) { return 0; }
}
