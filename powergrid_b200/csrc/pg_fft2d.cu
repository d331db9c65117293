// Oversampled 2-D FFTs for power-of-two grids (2N x 2N, N = 32 ... 512),
// written as four pruned passes with the pre- and post-kernels fused in.
//
// The forward operator's input grid is zero outside the N x N image region
// (zero_pad, griddingSupport.cpp:372-404) and the adjoint keeps only that
// region of its output (crop_center_region, :408-460).  cuFFT transforms the
// whole grid twice per direction; here
//   forward  F1  per image row: pre-kernel values (deapodization, coil map,
//                shot and segment phases, checkerboard sign) into a zero-
//                padded row, FFT along y                      -> N rows
//            F2  per grid column: the N nonzero rows, zero padded, FFT along
//                x                                             -> full grid
//   adjoint  A1  per grid column: inverse FFT along x, keep the N cropped rows
//            A2  per cropped row: inverse FFT along y, keep the N cropped
//                columns, post-kernel weights (sign, deapodization, WoH,
//                conj coil map, conj shot phase)               -> one image per grid
//            sum the images of the batch's grids in a fixed order.
// Transforms are unnormalised (FFTW/cuFFT conventions, forward sign -1) and
// run in shared memory as Stockham radix-4 (+ one radix-2) passes over a
// batch of rows; twiddles come from a table made in double precision.
#include <cmath>
#include <vector>

#include "pg_fft2d.cuh"

namespace pg {
namespace {

constexpr int kThreads = 256;
constexpr int kElems = 2048;   // complex values per block and buffer

__device__ __forceinline__ float2 twiddle(float2 v, float2 w, bool inv) {
  const float wy = inv ? -w.y : w.y;
  return make_float2(v.x * w.x - v.y * wy, v.x * wy + v.y * w.x);
}

// Row layout in shared memory: one padding element after every 16 (the
// radix-16 Stockham loads and stores then hit 16 distinct 8-byte bank pairs
// per half-warp), and a row stride of 2 (mod 16) elements, so the column
// kernels' transposed accesses (8 columns x 2 rows per half-warp at n = 256)
// are conflict-free too.
__host__ __device__ constexpr int pad16(int c) { return c + (c >> 4); }
template <int LOGN>
__host__ __device__ constexpr int row_stride() { return pad16(1 << LOGN) + 2; }

// exp(-/+ 2 pi i m / 16) * v for a compile-time m (constants of the unit circle).
template <int M>
__device__ __forceinline__ float2 rot16(float2 v, bool inv) {
  constexpr float kC[16] = {1.f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f, 0.f,
                            -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f, -1.f,
                            -0.92387953251128674f, -0.70710678118654752f, -0.38268343236508977f, 0.f,
                            0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f};
  constexpr float c = kC[M % 16];
  constexpr float sn = kC[(M + 12) % 16];   // sin(2 pi m/16) = cos(2 pi (m - 4)/16)
  const float sy = inv ? sn : -sn;
  return make_float2(v.x * c - v.y * sy, v.x * sy + v.y * c);
}

__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3, bool inv) {
  const float2 t0 = make_float2(v0.x + v2.x, v0.y + v2.y), t1 = make_float2(v0.x - v2.x, v0.y - v2.y);
  const float2 t2 = make_float2(v1.x + v3.x, v1.y + v3.y), t3 = make_float2(v1.x - v3.x, v1.y - v3.y);
  // -i*t3 = (t3.y, -t3.x)
  const float2 m3 = inv ? make_float2(-t3.y, t3.x) : make_float2(t3.y, -t3.x);
  v0 = make_float2(t0.x + t2.x, t0.y + t2.y);
  v1 = make_float2(t1.x + m3.x, t1.y + m3.y);
  v2 = make_float2(t0.x - t2.x, t0.y - t2.y);
  v3 = make_float2(t1.x - m3.x, t1.y - m3.y);
}

// 16-point DFT in registers as 4 x 4: y[k1 + 4 k2] = sum_n2 W4^(n2 k2) W16^(n2 k1)
// sum_n1 W4^(n1 k1) v[4 n1 + n2].
__device__ __forceinline__ void dft16(float2 (&v)[16], bool inv) {
  dft4(v[0], v[4], v[8], v[12], inv);
  dft4(v[1], v[5], v[9], v[13], inv);
  dft4(v[2], v[6], v[10], v[14], inv);
  dft4(v[3], v[7], v[11], v[15], inv);
  // v[4 k1 + n2] now holds u[n2][k1]
  v[5] = rot16<1>(v[5], inv);   v[6] = rot16<2>(v[6], inv);   v[7] = rot16<3>(v[7], inv);
  v[9] = rot16<2>(v[9], inv);   v[10] = rot16<4>(v[10], inv); v[11] = rot16<6>(v[11], inv);
  v[13] = rot16<3>(v[13], inv); v[14] = rot16<6>(v[14], inv); v[15] = rot16<9>(v[15], inv);
  dft4(v[0], v[1], v[2], v[3], inv);
  dft4(v[4], v[5], v[6], v[7], inv);
  dft4(v[8], v[9], v[10], v[11], inv);
  dft4(v[12], v[13], v[14], v[15], inv);
  // v[4 k1 + k2] holds y[k1 + 4 k2]: transpose the 4 x 4 index
  float2 t;
  t = v[1]; v[1] = v[4]; v[4] = t;
  t = v[2]; v[2] = v[8]; v[8] = t;
  t = v[3]; v[3] = v[12]; v[12] = t;
  t = v[6]; v[6] = v[9]; v[9] = t;
  t = v[7]; v[7] = v[13]; v[13] = t;
  t = v[11]; v[11] = v[14]; v[14] = t;
}

// One Stockham pass of radix R (16, 4 or 2) over ROWS rows of length n,
// a -> b, after Ns = product of the earlier radices.
template <int LOGN, int ROWS, int R>
__device__ __forceinline__ void fft_stage(const float2* a, float2* b, int Ns, const float2* tw, bool inv) {
  constexpr int n = 1 << LOGN, m = n / R, RS = row_stride<LOGN>();
  constexpr int total = ROWS * m;
  constexpr int per = (total + kThreads - 1) / kThreads;
  const int step = n / (Ns * R);
#pragma unroll
  for (int it = 0; it < per; ++it) {
    const int idx = it * kThreads + threadIdx.x;
    if (total % kThreads != 0 && idx >= total) break;
    const int row = idx / m, j = idx % m;
    const float2* s = a + row * RS;
    float2* d = b + row * RS;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[pad16(j + r * m)];
    const int k = j & (Ns - 1);
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = twiddle(v[r], tw[r * k * step], inv);
    }
    if constexpr (R == 16) {
      dft16(v, inv);
    } else if constexpr (R == 4) {
      dft4(v[0], v[1], v[2], v[3], inv);
    } else {
      const float2 t = v[0];
      v[0] = make_float2(t.x + v[1].x, t.y + v[1].y);
      v[1] = make_float2(t.x - v[1].x, t.y - v[1].y);
    }
    const int o = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[pad16(o + r * Ns)] = v[r];
  }
  __syncthreads();
}

// Batched in-shared-memory FFT of ROWS rows of length n = 2^LOGN (row r at
// a + r*row_stride, padded by pad16); b is scratch of the same shape and tw
// the twiddle table (in shared memory).  Radix-16 passes, then one radix-4
// and/or radix-2 pass.  Returns the buffer that holds the result, in natural
// order.
template <int LOGN, int ROWS>
__device__ float2* fft_rows(float2* a, float2* b, const float2* tw, bool inv) {
  int Ns = 1;
#pragma unroll
  for (int st = 0; st < LOGN / 4; ++st) {
    fft_stage<LOGN, ROWS, 16>(a, b, Ns, tw, inv);
    float2* t = a; a = b; b = t;
    Ns *= 16;
  }
  if ((LOGN % 4) >= 2) {
    fft_stage<LOGN, ROWS, 4>(a, b, Ns, tw, inv);
    float2* t = a; a = b; b = t;
    Ns *= 4;
  }
  if (LOGN % 2) {
    fft_stage<LOGN, ROWS, 2>(a, b, Ns, tw, inv);
    float2* t = a; a = b; b = t;
  }
  return a;
}

// Copy the n-entry twiddle table into shared memory.
template <int LOGN>
__device__ __forceinline__ void load_twiddles(float2* stw, const float2* __restrict__ tw) {
  constexpr int n = 1 << LOGN;
#pragma unroll
  for (int it = 0; it < (n + kThreads - 1) / kThreads; ++it) {
    const int k = it * kThreads + threadIdx.x;
    if (k < n) stw[k] = tw[k];
  }
}

__device__ __forceinline__ int parity2(int a, int b) { return (a + b) & 1; }

// Shared memory per block: two R-row buffers and the twiddle table.
template <int LOGN>
constexpr size_t fft_smem_bytes() {
  return (2ull * (kElems / (1 << LOGN)) * row_stride<LOGN>() + (1 << LOGN)) * sizeof(float2);
}

// F1: pre-kernel values of image rows ix (R rows per block) of grid b,
// zero padded to n, FFT along y -> P[b][ix][0..n).
template <int LOGN>
__global__ void __launch_bounds__(kThreads) k_fft_fwd_rows(NufftGeom g, int L, const float2* __restrict__ x,
                                                           const float2* __restrict__ S, int c0,
                                                           const float2* __restrict__ E,
                                                           const float2* __restrict__ Wo,
                                                           const float* __restrict__ deapf,
                                                           const float2* __restrict__ tw, float2* __restrict__ P) {
  constexpr int n = 1 << LOGN, R = kElems / n, stride = row_stride<LOGN>(), PER = kElems / kThreads;
  extern __shared__ float2 sh[];
  float2* a = sh;
  float2* bb = sh + R * stride;
  float2* stw = sh + 2 * R * stride;
  load_twiddles<LOGN>(stw, tw);
  const int Nn = g.Ny, pad = g.pad_off[1];
  const uint64_t N = g.nimg();
  const int b = blockIdx.y, c = b / L, l = b - c * L;
  const int ix0 = blockIdx.x * R;
#pragma unroll
  for (int it = 0; it < PER; ++it) {
    const int e = it * kThreads + threadIdx.x;
    const int r = e / n, gy = e % n;
    const int ix = ix0 + r;
    float2 v = make_float2(0.f, 0.f);
    const int iy = gy - pad;
    if (ix < g.Nx && iy >= 0 && iy < Nn) {
      const uint64_t p = (uint64_t)iy + (uint64_t)Nn * ix;
      v = x[p];
      if (S) {
        const float2 sv = S[(uint64_t)(c0 + c) * N + p];
        v = E ? cmul(v, cmul(sv, E[p])) : cmul(sv, v);
      }
      if (Wo) v = cmul(Wo[(uint64_t)l * N + p], v);
      const float f = parity2(ix + g.pad_off[0], gy) ? -deapf[p] : deapf[p];
      v = make_float2(v.x * f, v.y * f);
    }
    a[r * stride + pad16(gy)] = v;
  }
  __syncthreads();
  const float2* res = fft_rows<LOGN, R>(a, bb, stw, false);
#pragma unroll
  for (int it = 0; it < PER; ++it) {
    const int e = it * kThreads + threadIdx.x;
    const int r = e / n, gy = e % n;
    if (ix0 + r < g.Nx) P[((uint64_t)b * g.Nx + ix0 + r) * n + gy] = res[r * stride + pad16(gy)];
  }
}

// F2: columns gy (R per block) of grid b: the Nx rows of P at gx = pad + i,
// zero padded to n, FFT along x -> grids[b][gx][gy] for every gx.
template <int LOGN>
__global__ void __launch_bounds__(kThreads) k_fft_fwd_cols(NufftGeom g, const float2* __restrict__ P,
                                                           const float2* __restrict__ tw,
                                                           float2* __restrict__ grids) {
  constexpr int n = 1 << LOGN, R = kElems / n, stride = row_stride<LOGN>(), PER = kElems / kThreads;
  extern __shared__ float2 sh[];
  float2* a = sh;
  float2* bb = sh + R * stride;
  float2* stw = sh + 2 * R * stride;
  load_twiddles<LOGN>(stw, tw);
  const int pad = g.pad_off[0];
  const int b = blockIdx.y, gy0 = blockIdx.x * R;
#pragma unroll
  for (int it = 0; it < PER; ++it) {
    const int e = it * kThreads + threadIdx.x;
    const int gx = e / R, cl = e % R;
    const int i = gx - pad;
    float2 v = make_float2(0.f, 0.f);
    if (i >= 0 && i < g.Nx) v = P[((uint64_t)b * g.Nx + i) * n + gy0 + cl];
    a[cl * stride + pad16(gx)] = v;
  }
  __syncthreads();
  const float2* res = fft_rows<LOGN, R>(a, bb, stw, false);
  const uint64_t G = (uint64_t)n * n;
#pragma unroll
  for (int it = 0; it < PER; ++it) {
    const int e = it * kThreads + threadIdx.x;
    const int gx = e / R, cl = e % R;
    grids[(uint64_t)b * G + (uint64_t)gx * n + gy0 + cl] = res[cl * stride + pad16(gx)];
  }
}

// A1: columns gy of grid b, inverse FFT along x, keep gx = crop + i -> Q[b][i][gy].
template <int LOGN>
__global__ void __launch_bounds__(kThreads) k_fft_inv_cols(NufftGeom g, const float2* __restrict__ grids,
                                                           const float2* __restrict__ tw, float2* __restrict__ Q) {
  constexpr int n = 1 << LOGN, R = kElems / n, stride = row_stride<LOGN>(), PER = kElems / kThreads;
  extern __shared__ float2 sh[];
  float2* a = sh;
  float2* bb = sh + R * stride;
  float2* stw = sh + 2 * R * stride;
  load_twiddles<LOGN>(stw, tw);
  const int crop = g.crop_off[0];
  const int b = blockIdx.y, gy0 = blockIdx.x * R;
  const uint64_t G = (uint64_t)n * n;
#pragma unroll
  for (int it = 0; it < PER; ++it) {
    const int e = it * kThreads + threadIdx.x;
    const int gx = e / R, cl = e % R;
    a[cl * stride + pad16(gx)] = grids[(uint64_t)b * G + (uint64_t)gx * n + gy0 + cl];
  }
  __syncthreads();
  const float2* res = fft_rows<LOGN, R>(a, bb, stw, true);
#pragma unroll
  for (int it = 0; it < PER / 2; ++it) {    // the Nx = n/2 cropped rows
    const int e = it * kThreads + threadIdx.x;
    const int i = e / R, cl = e % R;
    Q[((uint64_t)b * g.Nx + i) * n + gy0 + cl] = res[cl * stride + pad16(crop + i)];
  }
}

// A2: cropped rows ix of grid b, inverse FFT along y, keep gy = crop + iy and
// apply the post-kernel weights of grid b = (coil c, segment l) -> Rimg[b][p].
template <int LOGN>
__global__ void __launch_bounds__(kThreads) k_fft_inv_rows(NufftGeom g, int L, const float2* __restrict__ Q,
                                                           const float2* __restrict__ S, int c0,
                                                           const float2* __restrict__ E,
                                                           const float2* __restrict__ WoH,
                                                           const float* __restrict__ deapf,
                                                           const float2* __restrict__ tw,
                                                           float2* __restrict__ Rimg) {
  constexpr int n = 1 << LOGN, R = kElems / n, stride = row_stride<LOGN>(), PER = kElems / kThreads;
  extern __shared__ float2 sh[];
  float2* a = sh;
  float2* bb = sh + R * stride;
  float2* stw = sh + 2 * R * stride;
  load_twiddles<LOGN>(stw, tw);
  constexpr int Nn = n / 2;
  const int crop = g.crop_off[1];
  const uint64_t N = g.nimg();
  const int b = blockIdx.y, c = b / L, l = b - c * L;
  const int ix0 = blockIdx.x * R;
#pragma unroll
  for (int it = 0; it < PER; ++it) {
    const int e = it * kThreads + threadIdx.x;
    const int r = e / n, gy = e % n;
    float2 v = make_float2(0.f, 0.f);
    if (ix0 + r < g.Nx) v = Q[((uint64_t)b * g.Nx + ix0 + r) * n + gy];
    a[r * stride + pad16(gy)] = v;
  }
  __syncthreads();
  const float2* res = fft_rows<LOGN, R>(a, bb, stw, true);
#pragma unroll
  for (int it = 0; it < PER / 2; ++it) {    // the Ny = n/2 cropped columns of R rows
    const int e = it * kThreads + threadIdx.x;
    const int r = e / Nn, iy = e % Nn;
    const int ix = ix0 + r;
    if (ix >= g.Nx) continue;
    const uint64_t p = (uint64_t)iy + (uint64_t)Nn * ix;
    float2 v = res[r * stride + pad16(crop + iy)];
    const float f = parity2(ix + g.crop_off[0], iy + crop) ? -deapf[p] : deapf[p];
    v = make_float2(v.x * f, v.y * f);
    if (WoH) v = cmul(v, WoH[(uint64_t)l * N + p]);
    if (S) {
      const float2 sv = S[(uint64_t)(c0 + c) * N + p];
      v = E ? cmul(cmul(cconj(sv), cconj(E[p])), v) : cmul(v, cconj(sv));
    }
    Rimg[(uint64_t)b * N + p] = v;
  }
}

// x[p] (+)= sum over the batch's grids of Rimg[b][p]: 8 lanes per pixel, lane
// k takes grids k, k+8, ..., added by a fixed xor butterfly.
__global__ void k_sum_images(uint64_t N, int B, const float2* __restrict__ Rimg, int accumulate,
                             float2* __restrict__ x) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int k = (int)(t & 7);
  const uint64_t p = t >> 3;
  float2 acc = make_float2(0.f, 0.f);
  if (p < N)
    for (int b = k; b < B; b += 8) acc = cadd(acc, Rimg[(uint64_t)b * N + p]);
#pragma unroll
  for (int o = 4; o >= 1; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if (p < N && k == 0) x[p] = accumulate ? cadd(x[p], acc) : acc;
}

template <int LOGN>
pg_status forward_t(const NufftGeom& g, int B, int L, const float2* x, const float2* S, int c0, const float2* E,
                    const float2* Wo, const float* deapf, const float2* tw, float2* P, float2* grids,
                    cudaStream_t s) {
  constexpr int n = 1 << LOGN, R = kElems / n;
  const size_t smem = fft_smem_bytes<LOGN>();
  PG_CUDA(cudaFuncSetAttribute(k_fft_fwd_rows<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PG_CUDA(cudaFuncSetAttribute(k_fft_fwd_cols<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PG_LAUNCH(k_fft_fwd_rows<LOGN>, dim3(ceil_div(g.Nx, R), B), kThreads, smem, s, g, L, x, S, c0, E, Wo, deapf, tw, P);
  PG_LAUNCH(k_fft_fwd_cols<LOGN>, dim3(n / R, B), kThreads, smem, s, g, P, tw, grids);
  return PG_OK;
}

template <int LOGN>
pg_status adjoint_t(const NufftGeom& g, int B, int L, const float2* grids, const float2* S, int c0, const float2* E,
                    const float2* WoH, const float* deapf, const float2* tw, float2* Q, float2* Rimg,
                    cudaStream_t s) {
  constexpr int n = 1 << LOGN, R = kElems / n;
  const size_t smem = fft_smem_bytes<LOGN>();
  PG_CUDA(cudaFuncSetAttribute(k_fft_inv_cols<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PG_CUDA(cudaFuncSetAttribute(k_fft_inv_rows<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PG_LAUNCH(k_fft_inv_cols<LOGN>, dim3(n / R, B), kThreads, smem, s, g, grids, tw, Q);
  PG_LAUNCH(k_fft_inv_rows<LOGN>, dim3(ceil_div(g.Nx, R), B), kThreads, smem, s, g, L, Q, S, c0, E, WoH, deapf, tw,
            Rimg);
  return PG_OK;
}

int log2_exact(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return ((1 << l) == v) ? l : -1;
}

}  // namespace

bool fft2d_supported(const NufftGeom& g) {
  if (g.dim != 2 || g.Gx != g.Gy || g.Gx != 2 * g.Nx || g.Ny != g.Nx) return false;
  const int l = log2_exact(g.Gx);
  return l >= 6 && l <= 10;
}

pg_status fft2d_twiddles(const NufftGeom& g, DevBuf<float2>* tw, cudaStream_t s) {
  const int n = g.Gx;
  std::vector<float2> h(n);
  const double two_pi = 6.283185307179586476925286766559;
  for (int k = 0; k < n; ++k) {
    const double a = -two_pi * (double)k / (double)n;
    h[k] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  return tw->upload(h.data(), h.size(), s);
}

pg_status fft2d_forward(const NufftGeom& g, int B, int L, const float2* x, const float2* S, int c0, const float2* E,
                        const float2* Wo, const float* deapf, const float2* tw, float2* P, float2* grids,
                        cudaStream_t s) {
  switch (log2_exact(g.Gx)) {
    case 6: return forward_t<6>(g, B, L, x, S, c0, E, Wo, deapf, tw, P, grids, s);
    case 7: return forward_t<7>(g, B, L, x, S, c0, E, Wo, deapf, tw, P, grids, s);
    case 8: return forward_t<8>(g, B, L, x, S, c0, E, Wo, deapf, tw, P, grids, s);
    case 9: return forward_t<9>(g, B, L, x, S, c0, E, Wo, deapf, tw, P, grids, s);
    case 10: return forward_t<10>(g, B, L, x, S, c0, E, Wo, deapf, tw, P, grids, s);
  }
  return set_error(PG_INVALID_ARG, "fft2d: unsupported grid %d", g.Gx);
}

pg_status fft2d_adjoint(const NufftGeom& g, int B, int L, const float2* grids, const float2* S, int c0,
                        const float2* E, const float2* WoH, const float* deapf, const float2* tw, float2* Q,
                        float2* Rimg, int accumulate, float2* x, cudaStream_t s) {
  pg_status st = PG_INVALID_ARG;
  switch (log2_exact(g.Gx)) {
    case 6: st = adjoint_t<6>(g, B, L, grids, S, c0, E, WoH, deapf, tw, Q, Rimg, s); break;
    case 7: st = adjoint_t<7>(g, B, L, grids, S, c0, E, WoH, deapf, tw, Q, Rimg, s); break;
    case 8: st = adjoint_t<8>(g, B, L, grids, S, c0, E, WoH, deapf, tw, Q, Rimg, s); break;
    case 9: st = adjoint_t<9>(g, B, L, grids, S, c0, E, WoH, deapf, tw, Q, Rimg, s); break;
    case 10: st = adjoint_t<10>(g, B, L, grids, S, c0, E, WoH, deapf, tw, Q, Rimg, s); break;
    default: return set_error(PG_INVALID_ARG, "fft2d: unsupported grid %d", g.Gx);
  }
  if (st != PG_OK) return st;
  const uint64_t N = g.nimg();
  PG_LAUNCH(k_sum_images, ceil_div(N * 8, 256), 256, 0, s, N, B, Rimg, accumulate, x);
  return PG_OK;
}

}  // namespace pg
