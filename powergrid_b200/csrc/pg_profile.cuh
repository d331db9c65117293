// Stage tracing: NVTX ranges, and CUDA-event timing enabled on demand (see
// pg_profile_enable).
#pragma once

#include <nvtx3/nvToolsExt.h>

#include "pg_common.cuh"

namespace pg {

extern bool g_profile;
// Set while capturing a graph that must carry no stage events.
extern thread_local bool g_profile_suppress;
// Changes whenever the recording set changes (captured graphs embed it).
extern uint64_t g_profile_epoch;
// Record the start / stop event of `stage` on stream s (no-op unless enabled).
void prof_start(const char* stage, cudaStream_t s);
void prof_stop(const char* stage, cudaStream_t s);

// A stage: an NVTX range on the host (always; free without a tool attached)
// and, when stage timing is on, a CUDA event pair on the stream.
struct ProfScope {
  const char* name;
  cudaStream_t s;
  bool on;
  ProfScope(const char* n, cudaStream_t st) : name(n), s(st), on(g_profile && !g_profile_suppress) {
    nvtxRangePushA(name);
    if (on) prof_start(name, s);
  }
  ~ProfScope() {
    if (on) prof_stop(name, s);
    nvtxRangePop();
  }
};

}  // namespace pg
