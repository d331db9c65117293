// Stage timing with CUDA events (enabled on demand; see pg_profile_enable).
#pragma once

#include "pg_common.cuh"

namespace pg {

extern bool g_profile;
// Changes whenever the recording set changes (captured graphs embed it).
extern uint64_t g_profile_epoch;
// Record the start / stop event of `stage` on stream s (no-op unless enabled).
void prof_start(const char* stage, cudaStream_t s);
void prof_stop(const char* stage, cudaStream_t s);

struct ProfScope {
  const char* name;
  cudaStream_t s;
  ProfScope(const char* n, cudaStream_t st) : name(n), s(st) { if (g_profile) prof_start(name, s); }
  ~ProfScope() { if (g_profile) prof_stop(name, s); }
};

}  // namespace pg
