// Gdft forward without any device allocation.
//
// Some callers cannot let a library allocate device memory: applications that
// own every byte of device memory through their own pool or a fixed budget,
// and latency-critical pipelines that must not meet cudaMalloc's implicit
// device-wide synchronisation or an out-of-memory failure in the middle of a
// run.  For them pg_gdft_forward_noalloc computes y = Gdft * x for one coil
// from the caller's device buffers alone.  The only scratch it needs — the
// per-split partial sums of the sample sums — lives in a fixed file-scope
// device array instead of an allocated buffer.
//
// That array is 4 MiB (kNoAllocPartials complex values).  Every GPU that
// loads this library holds it until the process exits.  All calls share it:
// two calls whose work overlaps on the GPU (for example on two streams)
// race on it and must be ordered by the caller.  A call overwrites every
// partial it later reads, so nothing from an earlier call carries over and
// no clearing is needed.
//
// The call runs on the library's device (the one given to pg_init, which the
// library makes current); the caller's buffers must live on that device.
// In host code the array's name is only a host-side stand-in; the device
// address is obtained with cudaGetSymbolAddress, with that device current,
// on the first call after pg_init (pg_shutdown forgets it, so a call after
// a later pg_init looks it up again).  That first call should therefore
// happen before any stream capture.
#include <mutex>

#include "pg_gdft.cuh"

namespace pg {

namespace {

constexpr uint64_t kNoAllocPartials = 1ull << 19;  // 512 Ki complex64 = 4 MiB
constexpr int kTileNA = 128;

static __device__ __align__(256) float2 g_noalloc_partials[kNoAllocPartials];

std::mutex g_na_mu;
float2* g_na_addr = nullptr;  // device address of g_noalloc_partials on g_na_dev
int g_na_dev = -1;

__device__ __forceinline__ void na_phase_sincos(double ph, float* s, float* c) {
  const double inv2pi = 0.15915494309189533577;   // 1 / (2 pi)
  const double twopi = 6.283185307179586476925;    // 2 pi (double)
  const double n = rint(ph * inv2pi);
  const float r = (float)fma(-n, twopi, ph);      // |r| <= pi
  __sincosf(r, s, c);
}

// The forward DFT partial sums of k_dft_forward for one coil, reading the
// float trajectory, voxel coordinates, field map and times directly (the
// double-precision operands are formed on the fly exactly as the operator's
// set-up forms them), so no packed copies are needed.
__global__ void __launch_bounds__(kTileNA) k_dft_forward_noalloc(uint64_t nk, uint64_t ni,
    const float* __restrict__ kx, const float* __restrict__ ky, const float* __restrict__ kz,
    const float* __restrict__ t, const float* __restrict__ ix, const float* __restrict__ iy,
    const float* __restrict__ iz, const float* __restrict__ fm, const float2* __restrict__ x, uint64_t jchunk,
    float2* __restrict__ part) {
  __shared__ double4 sv[kTileNA];
  __shared__ float2 sx[kTileNA];
  const double tpi = 6.283185307179586476925;
  const uint64_t i = (uint64_t)blockIdx.x * kTileNA + threadIdx.x;
  const uint64_t j0 = (uint64_t)blockIdx.y * jchunk;
  const uint64_t j1 = (j0 + jchunk < ni) ? j0 + jchunk : ni;
  double4 k = make_double4(0, 0, 0, 0);
  if (i < nk) k = make_double4(tpi * (double)kx[i], tpi * (double)ky[i], tpi * (double)kz[i], (double)t[i]);
  float2 tot = make_float2(0.f, 0.f);
  for (uint64_t jt = j0; jt < j1; jt += kTileNA) {
    const int n = (int)((j1 - jt) < (uint64_t)kTileNA ? (j1 - jt) : (uint64_t)kTileNA);
    __syncthreads();
    if (threadIdx.x < n) {
      const uint64_t j = jt + threadIdx.x;
      sv[threadIdx.x] = make_double4((double)ix[j], (double)iy[j], (double)iz[j], (double)fm[j]);
      sx[threadIdx.x] = x[j];
    }
    __syncthreads();
    float2 acc = make_float2(0.f, 0.f);
    for (int j = 0; j < n; ++j) {
      const double4 v = sv[j];
      const double ph = fma(k.x, v.x, fma(k.y, v.y, fma(k.z, v.z, v.w * k.w)));
      float s, co;
      na_phase_sincos(ph, &s, &co);
      const float2 xv = sx[j];
      acc.x = fmaf(co, xv.x, fmaf(s, xv.y, acc.x));
      acc.y = fmaf(co, xv.y, fmaf(-s, xv.x, acc.y));
    }
    tot.x += acc.x;
    tot.y += acc.y;
  }
  if (i < nk) part[(uint64_t)blockIdx.y * nk + i] = tot;
}

// y[i] = sum over splits of part[q * nk + i], in split order.
__global__ void k_dft_finish_noalloc(uint64_t nk, int nsplit, const float2* __restrict__ part,
                                     float2* __restrict__ y) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nk) return;
  float2 s = part[i];
  for (int q = 1; q < nsplit; ++q) s = cadd(s, part[(uint64_t)q * nk + i]);
  y[i] = s;
}

// The scratch array's device address on the current (library) device.
pg_status noalloc_scratch(float2** out) {
  int dev = 0;
  PG_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_addr || g_na_dev != dev) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return set_error(PG_CUDA_ERROR, "no-alloc Gdft: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    }
    g_na_addr = static_cast<float2*>(p);
    g_na_dev = dev;
  }
  *out = g_na_addr;
  return PG_OK;
}

}  // namespace

// Called by pg_shutdown: the cached address belongs to the context that ends.
void noalloc_forget_scratch() {
  std::lock_guard<std::mutex> lk(g_na_mu);
  g_na_addr = nullptr;
  g_na_dev = -1;
}

}  // namespace pg

using namespace pg;

extern "C" {

pg_status pg_gdft_forward_noalloc(uint64_t nk, uint64_t ni, const float* kx, const float* ky, const float* kz,
                                  const float* ix, const float* iy, const float* iz, const float* field_map,
                                  const float* t, const void* x_dev, void* y_dev, void* stream) {
  if (!kx || !ky || !kz || !ix || !iy || !iz || !field_map || !t || !x_dev || !y_dev)
    return set_error(PG_INVALID_ARG, "no-alloc Gdft: null argument");
  if (nk == 0 || ni == 0) return set_error(PG_INVALID_ARG, "no-alloc Gdft: empty operator");
  if (nk > kNoAllocPartials)
    return set_error(PG_INVALID_ARG,
                     "no-alloc Gdft: %llu samples exceed the fixed scratch of %llu partial sums (4 MiB); "
                     "use pg_gdft_create / pg_op_forward_device for larger problems",
                     (unsigned long long)nk, (unsigned long long)kNoAllocPartials);
  PG_TRY(ensure_init());
  float2* part = nullptr;
  PG_TRY(noalloc_scratch(&part));
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  // split the voxel sum over blockIdx.y while the outputs alone do not fill
  // the GPU, as far as the fixed scratch allows
  const uint64_t blocks = (nk + kTileNA - 1) / kTileNA;
  uint64_t ns = ((uint64_t)sm_count() * 8 + blocks - 1) / blocks;
  const uint64_t max_inner = (ni + kTileNA - 1) / kTileNA;
  if (ns > max_inner) ns = max_inner;
  if (ns > 64) ns = 64;
  if (ns > kNoAllocPartials / nk) ns = kNoAllocPartials / nk;
  if (ns < 1) ns = 1;
  uint64_t jchunk = (ni + ns - 1) / ns;
  jchunk = (jchunk + kTileNA - 1) / kTileNA * kTileNA;
  dim3 grid((unsigned)blocks, (unsigned)ns);
  PG_LAUNCH(k_dft_forward_noalloc, grid, kTileNA, 0, s, nk, ni, kx, ky, kz, t, ix, iy, iz, field_map,
            (const float2*)x_dev, jchunk, part);
  PG_LAUNCH(k_dft_finish_noalloc, ceil_div(nk, 256), 256, 0, s, nk, (int)ns, part, (float2*)y_dev);
  return PG_OK;
}

}  // extern "C"
