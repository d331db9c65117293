// Shared infrastructure of the sm_100a library: status/error plumbing,
// device buffers with an allocation-failure hook, complex helpers and the
// kernel-launch counter.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "powergrid_b200.h"

namespace pg {

pg_status set_error(pg_status s, const char* fmt, ...);
// Drops the cached device address of the allocation-free Gdft's scratch array
// (pg_noalloc.cu); pg_shutdown calls it.
void noalloc_forget_scratch();
pg_status ensure_init();
cudaStream_t default_stream();
int sm_count();

// Counts this library's kernel launches (reported by bench.py).
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Host-side fault injection: the n-th allocation from the arm point fails.
extern std::atomic<uint64_t> g_fail_alloc_countdown;

pg_status dev_alloc(void** p, size_t bytes);
void dev_free(void* p);

// Per-thread device arena.  While a thread has an arena installed, device
// allocations are carved from one slab (falling back to stream-ordered pool
// allocations past its end) and frees are deferred to arena_release(), which
// returns everything stream-ordered on the arena's stream.  The request
// server uses one arena per request so that building and running a request
// never calls cudaMalloc/cudaFree, which would serialise the other streams.
struct Arena {
  char* base = nullptr;
  size_t cap = 0, used = 0;
  cudaStream_t stream = nullptr;
  std::vector<void*> overflow;
};
pg_status arena_open(Arena* a, size_t bytes, cudaStream_t s);
void arena_install(Arena* a);   // nullptr uninstalls
Arena* arena_current();
void arena_release(Arena* a);   // after all work on a->stream that uses it

#define PG_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) {                                                                       \
      cudaGetLastError(); /* do not leave a non-sticky error for the caller's next launch */      \
      return ::pg::set_error(PG_CUDA_ERROR, "%s:%d %s: %s", __FILE__, __LINE__, #call,            \
                             cudaGetErrorString(e_));                                              \
    }                                                                                              \
  } while (0)

#define PG_CUFFT(call)                                                                             \
  do {                                                                                             \
    cufftResult r_ = (call);                                                                       \
    if (r_ != CUFFT_SUCCESS)                                                                       \
      return ::pg::set_error(PG_CUFFT_ERROR, "%s:%d %s: cufft error %d", __FILE__, __LINE__, #call, \
                             (int)r_);                                                             \
  } while (0)

#define PG_TRY(call)                \
  do {                              \
    pg_status s_ = (call);          \
    if (s_ != PG_OK) return s_;     \
  } while (0)

// Programmatic dependent launch, for the kernels of a PCG iteration: the
// launch of the next kernel overlaps the previous kernel's completion.  A
// kernel launched this way calls pdl_wait() before it touches memory; the
// wait returns once the previous kernel has completed and its writes are
// visible (for a kernel launched without the attribute it returns at once).
// No kernel triggers its dependents early: successors' blocks resident next
// to a running kernel measured slower than the launch gap they hide.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// PG_NO_PDL=1 launches those kernels in plain stream order (read once).
bool pdl_enabled();

#define PG_LAUNCH_PDL(kernel, grid, block, smem, strm_, ...)                                       \
  do {                                                                                             \
    cudaLaunchConfig_t cfg_ = {};                                                                  \
    cfg_.gridDim = dim3(grid);                                                                     \
    cfg_.blockDim = dim3(block);                                                                   \
    cfg_.dynamicSmemBytes = (smem);                                                                \
    cfg_.stream = (strm_);                                                                         \
    cudaLaunchAttribute at_[1];                                                                    \
    at_[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;                                \
    at_[0].val.programmaticStreamSerializationAllowed = ::pg::pdl_enabled() ? 1 : 0;               \
    cfg_.attrs = at_;                                                                              \
    cfg_.numAttrs = 1;                                                                             \
    cudaError_t e_ = cudaLaunchKernelEx(&cfg_, kernel, __VA_ARGS__);                               \
    ::pg::count_launch();                                                                          \
    if (e_ != cudaSuccess) {                                                                       \
      cudaGetLastError();                                                                          \
      return ::pg::set_error(PG_CUDA_ERROR, "%s:%d launch %s: %s", __FILE__, __LINE__, #kernel,    \
                             cudaGetErrorString(e_));                                              \
    }                                                                                              \
  } while (0)

// ---- device-side index checks (PG_CHECKS builds) --------------------------
// Built with -DPG_CHECKS (libpowergrid_b200_checks.so), the gridding kernels
// check the indices their shared-memory and global accesses derive from the
// binning — window starts inside the tile, sample counts within the staging
// size, permutation entries inside the data — and, instead of accessing out of
// bounds or trapping, record the first failure in a device word of their
// translation unit and skip the access.  The record is (site << 48) | (low 48
// bits of the offending value); pg_checks_read returns and clears it.  In the
// product build PG_CHECK(...) is the constant true and the checks vanish.
enum pg_check_site {
  PG_SITE_SPREAD_COUNT = 1,    // item sample count > staging size
  PG_SITE_SPREAD_WINDOW = 2,   // sample window start outside its tile (k_spread)
  PG_SITE_SPREAD2D_WINDOW = 3, // run window start outside its tile (k_spread2d)
  PG_SITE_SPREAD2D_PERM = 4,   // permutation entry outside the data (k_spread2d)
  PG_SITE_GATHER_WINDOW = 5,   // sample window start outside its tile (k_gather)
  PG_SITE_GATHER_PERM = 6,     // permutation entry outside the data (k_gather)
};
// Host side: every translation unit with checks registers a reader of its word.
int register_check_reader(bool (*reader)(uint64_t* record));
#ifdef PG_CHECKS
__device__ __forceinline__ bool check_fail(unsigned long long* word, int site, long long v) {
  atomicCAS(word, 0ull, ((unsigned long long)site << 48) | ((unsigned long long)v & 0xffffffffffffull));
  return false;
}
#define PG_DEFINE_CHECK_WORD()                                                                     \
  static __device__ unsigned long long pg_check_word_;                                             \
  static bool pg_check_reader_(uint64_t* record) {                                                 \
    unsigned long long v = 0, zero = 0;                                                            \
    if (cudaMemcpyFromSymbol(&v, pg_check_word_, sizeof(v)) != cudaSuccess ||                      \
        cudaMemcpyToSymbol(pg_check_word_, &zero, sizeof(zero)) != cudaSuccess) {                  \
      cudaGetLastError();                                                                          \
      return false;                                                                                \
    }                                                                                              \
    *record = v;                                                                                   \
    return true;                                                                                   \
  }                                                                                                \
  static const int pg_check_registered_ = ::pg::register_check_reader(&pg_check_reader_);
#define PG_CHECK(cond, site, val) ((cond) || ::pg::check_fail(&pg_check_word_, (site), (long long)(val)))
#else
#define PG_DEFINE_CHECK_WORD()
#define PG_CHECK(cond, site, val) true
#endif

// Kernel launch followed by a launch-error check.
#define PG_LAUNCH(kernel, grid, block, smem, stream, ...)                                          \
  do {                                                                                             \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                                    \
    ::pg::count_launch();                                                                          \
    cudaError_t e_ = cudaGetLastError();                                                           \
    if (e_ != cudaSuccess)                                                                         \
      return ::pg::set_error(PG_CUDA_ERROR, "%s:%d launch %s: %s", __FILE__, __LINE__, #kernel,    \
                             cudaGetErrorString(e_));                                              \
  } while (0)

// Device buffer: owning, or a borrowed view of another buffer (borrow()),
// which the owner must outlive.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  bool owned = true;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), owned(o.owned) { o.p = nullptr; o.n = 0; o.owned = true; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      reset();
      p = o.p; n = o.n; owned = o.owned;
      o.p = nullptr; o.n = 0; o.owned = true;
    }
    return *this;
  }
  ~DevBuf() { reset(); }
  void reset() {
    if (p && owned) dev_free(p);
    p = nullptr;
    n = 0;
    owned = true;
  }
  void borrow(const DevBuf& o) {
    reset();
    p = o.p;
    n = o.n;
    owned = false;
  }
  pg_status alloc(size_t count) {
    if (count == n && p && owned) return PG_OK;
    reset();
    if (count == 0) return PG_OK;
    void* q = nullptr;
    PG_TRY(dev_alloc(&q, count * sizeof(T)));
    p = static_cast<T*>(q);
    n = count;
    return PG_OK;
  }
  pg_status upload(const T* host, size_t count, cudaStream_t s) {
    PG_TRY(alloc(count));
    if (count) PG_CUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    return PG_OK;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Grow a lazily-sized workspace used on stream s: queued work on s may still
// read the old buffer, so drain s before replacing it.
template <typename T>
inline pg_status grow(DevBuf<T>& b, size_t count, cudaStream_t s) {
  if (b.n >= count && b.p && b.owned) return PG_OK;
  if (b.p) PG_CUDA(cudaStreamSynchronize(s));
  return b.alloc(count);
}

// ---- complex helpers (float2 = interleaved complex64) ----------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

inline unsigned ceil_div(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace pg
