// Library context: device selection, default stream, error strings,
// allocation (with a host-side failure hook) and launch counting.
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "pg_common.cuh"

namespace pg {

std::atomic<uint64_t> g_launches{0};
std::atomic<uint64_t> g_fail_alloc_countdown{0};

namespace {
std::vector<bool (*)(uint64_t*)>& check_readers() {
  static std::vector<bool (*)(uint64_t*)> r;
  return r;
}
}  // namespace

int register_check_reader(bool (*reader)(uint64_t* record)) {
  check_readers().push_back(reader);
  return 0;
}

bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("PG_NO_PDL");
    return !(e && e[0] == '1');
  }();
  return on;
}

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
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, g_device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
  }
  PG_CUDA(cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking));
  g_inited = true;
  return PG_OK;
}

cudaStream_t default_stream() { return g_stream; }
int sm_count() { return g_sms; }

namespace {
thread_local Arena* t_arena = nullptr;
}

void arena_install(Arena* a) { t_arena = a; }
Arena* arena_current() { return t_arena; }

pg_status arena_open(Arena* a, size_t bytes, cudaStream_t s) {
  a->stream = s;
  a->cap = bytes;
  a->used = 0;
  a->overflow.clear();
  a->base = nullptr;
  if (bytes == 0) return PG_OK;
  cudaError_t e = cudaMallocAsync((void**)&a->base, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    a->base = nullptr;
    return set_error(e == cudaErrorMemoryAllocation ? PG_OUT_OF_MEMORY : PG_CUDA_ERROR,
                     "arena of %zu bytes: %s", bytes, cudaGetErrorString(e));
  }
  // make the slab usable from every stream before anything is carved from it
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) { cudaGetLastError(); return set_error(PG_CUDA_ERROR, "arena sync: %s", cudaGetErrorString(e)); }
  return PG_OK;
}

void arena_release(Arena* a) {
  if (a->base) cudaFreeAsync(a->base, a->stream);
  for (void* p : a->overflow) cudaFreeAsync(p, a->stream);
  a->base = nullptr;
  a->overflow.clear();
  a->cap = a->used = 0;
}

pg_status dev_alloc(void** p, size_t bytes) {
  if (t_arena) {
    Arena* a = t_arena;
    const size_t off = (a->used + 255) & ~size_t(255);
    if (a->base && off + bytes <= a->cap) {
      *p = a->base + off;
      a->used = off + bytes;
      return PG_OK;
    }
    cudaError_t e = cudaMallocAsync(p, bytes, a->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return set_error(PG_OUT_OF_MEMORY, "arena overflow allocation of %zu bytes failed", bytes);
    }
    a->overflow.push_back(*p);
    return PG_OK;
  }
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

void dev_free(void* p) {
  if (Arena* a = t_arena) {
    // arena memory is returned by arena_release
    if (a->base && (char*)p >= a->base && (char*)p < a->base + a->cap) return;
    for (void* q : a->overflow)
      if (q == p) return;
  }
  cudaFree(p);
}

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
  pg::noalloc_forget_scratch();
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

pg_status pg_checks_read(uint64_t* record, int* enabled) {
  if (!record || !enabled) return pg::set_error(PG_INVALID_ARG, "checks: null argument");
#ifdef PG_CHECKS
  *enabled = 1;
#else
  *enabled = 0;
#endif
  *record = 0;
  PG_TRY(pg::ensure_init());
  PG_CUDA(cudaDeviceSynchronize());
  for (auto* rd : pg::check_readers()) {
    uint64_t v = 0;
    if (!rd(&v)) return pg::set_error(PG_CUDA_ERROR, "checks: reading the device record failed");
    if (*record == 0) *record = v;
  }
  return PG_OK;
}

void pg_debug_fail_allocation_after(uint64_t n) { pg::g_fail_alloc_countdown.store(n); }

}  // extern "C"
