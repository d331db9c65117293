// Library context: device selection, default stream, error strings,
// allocation (with a host-side failure hook) and launch counting.
#include <cstring>
#include <mutex>

#include "pg_common.cuh"

namespace pg {

std::atomic<uint64_t> g_launches{0};
std::atomic<uint64_t> g_fail_alloc_countdown{0};

namespace {
thread_local std::string t_last_error;
std::mutex g_init_mu;
bool g_inited = false;
int g_device = 0;
int g_sms = 148;
cudaStream_t g_stream = nullptr;
}  // namespace

pg_status set_error(pg_status s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_last_error = buf;
  return s;
}

pg_status ensure_init() {
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (g_inited) {
    // keep the library device current for this host thread
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != g_device) PG_CUDA(cudaSetDevice(g_device));
    return PG_OK;
  }
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return set_error(PG_CUDA_ERROR, "no CUDA device available (%s)", cudaGetErrorString(e));
  if (g_device >= n) return set_error(PG_INVALID_ARG, "device %d out of range (%d devices)", g_device, n);
  PG_CUDA(cudaSetDevice(g_device));
  cudaDeviceProp prop;
  PG_CUDA(cudaGetDeviceProperties(&prop, g_device));
  if (prop.major < 10)
    return set_error(PG_CUDA_ERROR, "device %d is sm_%d%d; this library is built for sm_100a", g_device, prop.major,
                     prop.minor);
  g_sms = prop.multiProcessorCount;
  PG_CUDA(cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking));
  g_inited = true;
  return PG_OK;
}

cudaStream_t default_stream() { return g_stream; }
int sm_count() { return g_sms; }

pg_status dev_alloc(void** p, size_t bytes) {
  uint64_t c = g_fail_alloc_countdown.load();
  while (c > 0) {
    if (g_fail_alloc_countdown.compare_exchange_weak(c, c - 1)) {
      if (c == 1) return set_error(PG_OUT_OF_MEMORY, "injected allocation failure (%zu bytes)", bytes);
      break;
    }
  }
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return set_error(PG_OUT_OF_MEMORY, "cudaMalloc(%zu) failed: out of device memory", bytes);
  }
  if (e != cudaSuccess) return set_error(PG_CUDA_ERROR, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  return PG_OK;
}

void dev_free(void* p) { cudaFree(p); }

}  // namespace pg

extern "C" {

pg_status pg_init(int device) {
  {
    std::lock_guard<std::mutex> lk(pg::g_init_mu);
    if (pg::g_inited && device != pg::g_device)
      return pg::set_error(PG_INVALID_ARG, "already initialised on device %d", pg::g_device);
    pg::g_device = device;
  }
  return pg::ensure_init();
}

pg_status pg_shutdown(void) {
  std::lock_guard<std::mutex> lk(pg::g_init_mu);
  if (!pg::g_inited) return PG_OK;
  cudaStreamSynchronize(pg::g_stream);
  cudaStreamDestroy(pg::g_stream);
  pg::g_stream = nullptr;
  pg::g_inited = false;
  return PG_OK;
}

const char* pg_status_string(pg_status s) {
  switch (s) {
    case PG_OK: return "PG_OK";
    case PG_INVALID_ARG: return "PG_INVALID_ARG";
    case PG_OUT_OF_MEMORY: return "PG_OUT_OF_MEMORY";
    case PG_CUDA_ERROR: return "PG_CUDA_ERROR";
    case PG_TIMEOUT: return "PG_TIMEOUT";
    case PG_CANCELLED: return "PG_CANCELLED";
    case PG_NOT_INITIALIZED: return "PG_NOT_INITIALIZED";
    case PG_CUFFT_ERROR: return "PG_CUFFT_ERROR";
    case PG_REJECTED: return "PG_REJECTED";
    case PG_NOT_READY: return "PG_NOT_READY";
  }
  return "PG_UNKNOWN";
}

const char* pg_last_error(void) { return pg::t_last_error.c_str(); }

uint64_t pg_kernel_launch_count(void) { return pg::g_launches.load(); }

void pg_debug_fail_allocation_after(uint64_t n) { pg::g_fail_alloc_countdown.store(n); }

}  // extern "C"
