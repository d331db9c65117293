// Stage timing registry: one reusable event pair per stage name.
#include <map>
#include <mutex>
#include <string>

#include "pg_profile.cuh"

namespace pg {

bool g_profile = false;
thread_local bool g_profile_suppress = false;
uint64_t g_profile_epoch = 0;

namespace {
struct Pair {
  cudaEvent_t a = nullptr, b = nullptr;
  bool recorded = false;
};
std::mutex g_mu;
std::map<std::string, Pair> g_pairs;
std::string g_only;   // record only this stage when non-empty

Pair& get(const char* stage) {
  Pair& p = g_pairs[stage];
  if (!p.a) {
    cudaEventCreate(&p.a);
    cudaEventCreate(&p.b);
  }
  return p;
}
}  // namespace

// Inside a stream capture an ordinary event record only becomes a graph
// dependency; cudaEventRecordExternal makes it a record node that fires on
// every replay, so stages inside captured PCG iterations stay timeable.
static void record(cudaEvent_t e, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cs);
  if (cs == cudaStreamCaptureStatusActive)
    cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
  else
    cudaEventRecord(e, s);
}

void prof_start(const char* stage, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_only.empty() && g_only != stage) return;
  record(get(stage).a, s);
}
void prof_stop(const char* stage, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_only.empty() && g_only != stage) return;
  Pair& p = get(stage);
  record(p.b, s);
  p.recorded = true;
}

}  // namespace pg

extern "C" {

pg_status pg_profile_enable(int on) {
  PG_TRY(pg::ensure_init());
  pg::g_profile = on != 0;
  ++pg::g_profile_epoch;
  return PG_OK;
}

pg_status pg_profile_only(const char* stage) {
  std::lock_guard<std::mutex> lk(pg::g_mu);
  pg::g_only = stage ? stage : "";
  ++pg::g_profile_epoch;
  return PG_OK;
}

pg_status pg_profile_stage_ms(const char* stage, float* ms) {
  if (!stage || !ms) return pg::set_error(PG_INVALID_ARG, "profile: null argument");
  std::lock_guard<std::mutex> lk(pg::g_mu);
  auto it = pg::g_pairs.find(stage);
  if (it == pg::g_pairs.end() || !it->second.recorded) return pg::set_error(PG_NOT_READY, "stage %s not recorded", stage);
  PG_CUDA(cudaEventElapsedTime(ms, it->second.a, it->second.b));
  return PG_OK;
}

}  // extern "C"
