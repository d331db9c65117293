// Oversampled 2-D and 3-D FFTs for power-of-two grids (2N per axis,
// N = 16 ... 512), written as pruned passes with the pre- and post-kernels
// fused in.
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
// In 3-D the first pass runs over the Nx*Nz image lines along y, the second
// along x over each of the Nz nonzero z-slabs, and a third along z over every
// (x, y) column, reading only the Nz nonzero slabs; the adjoint mirrors it
// (z, keeping Nz slabs; x per slab, keeping Nx rows; y with the post weights).
// Transforms are unnormalised (FFTW/cuFFT conventions, forward sign -1).
//
// Each length-n transform (n = R1 * R2) is two register passes with one
// shared-memory transpose between them (the four-step form): with
// m = R2*m1 + m2 and k = k1 + R1*k2,
//   X[k] = sum_m2 W_R2^(m2 k2) * W_n^(m2 k1) * sum_m1 W_R1^(m1 k1) x[m].
// Pass 1: a thread takes one m2, loads its R1 inputs straight from global
// memory (consecutive threads: consecutive m2 or columns, so the loads
// coalesce), does the R1-point DFT in registers and the twiddle W_n^(m2 k1),
// and stores into shared memory.  Pass 2: a thread takes one k1, reads its R2
// values, does the R2-point DFT and stores X[k1 + R1 k2] straight to global
// memory.  Zero inputs (the padding) are never loaded and cropped outputs
// never stored.  Twiddles W_n^(m2 k1) come from a table made in double
// precision, laid out [k1][m2].
#include <algorithm>
#include <cmath>
#include <vector>

#include <cooperative_groups.h>

#include "pg_fftpass.cuh"

namespace cg = cooperative_groups;

namespace pg {
namespace {

constexpr int kT = 256;   // threads per block
constexpr int kMaxGridY = 65535;

__device__ __forceinline__ float2 twiddle(float2 v, float2 w, bool inv) {
  const float wy = inv ? -w.y : w.y;
  return make_float2(v.x * w.x - v.y * wy, v.x * wy + v.y * w.x);
}

// cos(2 pi m / 32), m = 0 .. 31 (points of the unit circle).
__device__ constexpr float kC32[32] = {
    1.f, 0.98078528040323044913f, 0.92387953251128675613f, 0.83146961230254523708f, 0.70710678118654752440f,
    0.55557023301960222474f, 0.38268343236508977173f, 0.19509032201612826785f, 0.f, -0.19509032201612826785f,
    -0.38268343236508977173f, -0.55557023301960222474f, -0.70710678118654752440f, -0.83146961230254523708f,
    -0.92387953251128675613f, -0.98078528040323044913f, -1.f, -0.98078528040323044913f, -0.92387953251128675613f,
    -0.83146961230254523708f, -0.70710678118654752440f, -0.55557023301960222474f, -0.38268343236508977173f,
    -0.19509032201612826785f, 0.f, 0.19509032201612826785f, 0.38268343236508977173f, 0.55557023301960222474f,
    0.70710678118654752440f, 0.83146961230254523708f, 0.92387953251128675613f, 0.98078528040323044913f};

// exp(-/+ 2 pi i m / 32) * v for a compile-time m.
template <int M>
__device__ __forceinline__ float2 rot32(float2 v, bool inv) {
  if constexpr (M % 32 == 0) {
    return v;
  } else {
    constexpr float c = kC32[M % 32];
    constexpr float sn = kC32[(M + 24) % 32];   // sin(2 pi m/32) = cos(2 pi (m - 8)/32)
    const float sy = inv ? sn : -sn;
    return make_float2(v.x * c - v.y * sy, v.x * sy + v.y * c);
  }
}

__device__ __forceinline__ void dft2(float2& a, float2& b) {
  const float2 t = a;
  a = make_float2(t.x + b.x, t.y + b.y);
  b = make_float2(t.x - b.x, t.y - b.y);
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

// 8-point DFT, natural order in and out: m = 2 m1 + m2, k = k1 + 4 k2.
__device__ __forceinline__ void dft8(float2 (&v)[8], bool inv) {
  dft4(v[0], v[2], v[4], v[6], inv);
  dft4(v[1], v[3], v[5], v[7], inv);
  v[3] = rot32<4>(v[3], inv);
  v[5] = rot32<8>(v[5], inv);
  v[7] = rot32<12>(v[7], inv);
  float2 y[8];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    float2 a = v[2 * k1], b = v[2 * k1 + 1];
    dft2(a, b);
    y[k1] = a;
    y[k1 + 4] = b;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = y[i];
}

// 16-point DFT as 4 x 4, natural order in and out.
__device__ __forceinline__ void dft16(float2 (&v)[16], bool inv) {
  dft4(v[0], v[4], v[8], v[12], inv);
  dft4(v[1], v[5], v[9], v[13], inv);
  dft4(v[2], v[6], v[10], v[14], inv);
  dft4(v[3], v[7], v[11], v[15], inv);
  // v[4 k1 + n2] now holds u[n2][k1]
  v[5] = rot32<2>(v[5], inv);   v[6] = rot32<4>(v[6], inv);   v[7] = rot32<6>(v[7], inv);
  v[9] = rot32<4>(v[9], inv);   v[10] = rot32<8>(v[10], inv); v[11] = rot32<12>(v[11], inv);
  v[13] = rot32<6>(v[13], inv); v[14] = rot32<12>(v[14], inv); v[15] = rot32<18>(v[15], inv);
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

template <int M>
__device__ __forceinline__ void rot_odd32(float2 (&o)[16], bool inv) {
  if constexpr (M < 16) {
    o[M] = rot32<M>(o[M], inv);
    rot_odd32<M + 1>(o, inv);
  }
}

// 32-point DFT as 16 x 2, natural order in and out: m = 2 m1 + m2, k = k1 + 16 k2.
__device__ __forceinline__ void dft32(float2 (&v)[32], bool inv) {
  float2 e[16], o[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
  dft16(e, inv);
  dft16(o, inv);
  rot_odd32<1>(o, inv);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    float2 a = e[k], b = o[k];
    dft2(a, b);
    v[k] = a;
    v[k + 16] = b;
  }
}

template <int R>
__device__ __forceinline__ void dft(float2 (&v)[R], bool inv) {
  if constexpr (R == 4) {
    dft4(v[0], v[1], v[2], v[3], inv);
  } else if constexpr (R == 8) {
    dft8(v, inv);
  } else if constexpr (R == 16) {
    dft16(v, inv);
  } else {
    static_assert(R == 32, "radix");
    dft32(v, inv);
  }
}

// Factor n = R1 * R2 of each supported length.
template <int LOGN> struct Split;
template <> struct Split<4> { static constexpr int R1 = 4, R2 = 4; };
template <> struct Split<5> { static constexpr int R1 = 8, R2 = 4; };
template <> struct Split<6> { static constexpr int R1 = 16, R2 = 4; };
template <> struct Split<7> { static constexpr int R1 = 16, R2 = 8; };
template <> struct Split<8> { static constexpr int R1 = 16, R2 = 16; };
template <> struct Split<9> { static constexpr int R1 = 16, R2 = 32; };
template <> struct Split<10> { static constexpr int R1 = 32, R2 = 32; };

// Row kernels: RB = kT / R2 rows per block.  Shared layout [row][k1][m2] with
// m2 stride R2 + 1 (odd: pass 2's threads, one k1 each, hit distinct banks)
// and a row stride = R2 (mod 16) (pass 1's half-warps span 16 / R2 rows).
template <int LOGN>
struct RowGeo {
  static constexpr int R1 = Split<LOGN>::R1, R2 = Split<LOGN>::R2, n = R1 * R2;
  static constexpr int RB = kT / R2;
  static constexpr int S2 = R2 + 1;
  static constexpr int base = R1 * S2;
  static constexpr int RS = base + (((R2 - base) % 16) + 16) % 16;
  static constexpr size_t smem = (size_t)RB * RS * sizeof(float2);
};

// Strided-line kernels: CB adjacent columns per block, shared layout [k1][m2][col].
template <int LOGN>
struct ColGeo {
  static constexpr int R1 = Split<LOGN>::R1, R2 = Split<LOGN>::R2, n = R1 * R2;
  static constexpr int CB = (4096 / n) > 8 ? (4096 / n) : 8;
  static constexpr size_t smem = (size_t)n * CB * sizeof(float2);
};

// A batch of strided lines: grid (or slab) b holds ncols columns; element
// m of column c sits at b * bstride + m * rstride + c.
struct Lines {
  uint64_t in_bstride, out_bstride, rstride;
  int ncols;
  int nio;      // nonzero input rows (forward) / kept output rows (inverse)
  int off;      // their first index along the line (pad / crop offset)
};

__device__ __forceinline__ int parity2(int a, int b) { return (a + b) & 1; }

// F1: pre-kernel values of the image lines (ix, iz) of grid b, zero padded
// to n along y, FFT along y -> P[b][iz][ix][0..n).
template <int LOGN>
__global__ void __launch_bounds__(kT) k_fft_fwd_rows(NufftGeom g, int L, const float2* __restrict__ x,
                                                     const float2* __restrict__ S, int c0,
                                                     const float2* __restrict__ E, const float2* __restrict__ Wo,
                                                     const float* __restrict__ deapf, const float2* __restrict__ tw,
                                                     float2* __restrict__ P) {
  pdl_wait();
  using RG = RowGeo<LOGN>;
  constexpr int R1 = RG::R1, R2 = RG::R2, n = RG::n, RB = RG::RB, S2 = RG::S2, RS = RG::RS;
  extern __shared__ float2 sh[];
  const int Nn = g.Ny, pad = g.pad_off[1];
  const int nrows = g.Nx * g.Nz;
  const uint64_t N = g.nimg();
  const int b = blockIdx.y, c = b / L, l = b - c * L;
  const int r0 = blockIdx.x * RB;
  {
    const int m2 = threadIdx.x % R2, r = threadIdx.x / R2;
    const int rg = r0 + r;
    const int ix = rg % g.Nx, iz = rg / g.Nx;
    const int pxz = ix + g.pad_off[0] + iz + g.pad_off[2];
    float2 v[R1];
#pragma unroll
    for (int m1 = 0; m1 < R1; ++m1) {
      const int gy = R2 * m1 + m2;
      const int iy = gy - pad;
      float2 u = make_float2(0.f, 0.f);
      if (rg < nrows && iy >= 0 && iy < Nn) {
        const uint64_t p = (uint64_t)iy + (uint64_t)Nn * ((uint64_t)ix + (uint64_t)g.Nx * iz);
        u = x[p];
        if (S) {
          const float2 sv = S[(uint64_t)(c0 + c) * N + p];
          u = E ? cmul(u, cmul(sv, E[p])) : cmul(sv, u);
        }
        if (Wo) u = cmul(Wo[(uint64_t)l * N + p], u);
        const float f = parity2(pxz, gy) ? -deapf[p] : deapf[p];
        u = make_float2(u.x * f, u.y * f);
      }
      v[m1] = u;
    }
    dft<R1>(v, false);
    float2* d = sh + r * RS + m2;
    d[0] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1) d[k1 * S2] = twiddle(v[k1], tw[k1 * R2 + m2], false);
  }
  __syncthreads();
#pragma unroll
  for (int it0 = 0; it0 < RB * R1; it0 += kT) {
    const int it = it0 + threadIdx.x;
    if ((RB * R1) % kT != 0 && it >= RB * R1) break;
    const int k1 = it % R1, r = it / R1;
    const int rg = r0 + r;
    float2 u[R2];
    const float2* s = sh + r * RS + k1 * S2;
#pragma unroll
    for (int m2 = 0; m2 < R2; ++m2) u[m2] = s[m2];
    dft<R2>(u, false);
    if (rg < nrows) {
      float2* o = P + ((uint64_t)b * nrows + rg) * n + k1;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) o[R1 * k2] = u[k2];
    }
  }
}

// Forward strided lines: per column, the nio nonzero rows at off + i
// (zero padded to n), FFT along the line -> all n rows of the output.
template <int LOGN>
__global__ void __launch_bounds__(kT) k_fft_fwd_cols(Lines ln, const float2* __restrict__ P,
                                                     const float2* __restrict__ tw, float2* __restrict__ out) {
  pdl_wait();
  using CG = ColGeo<LOGN>;
  constexpr int R1 = CG::R1, R2 = CG::R2, CB = CG::CB;
  extern __shared__ float2 sh[];
  const int b = blockIdx.y, c0 = blockIdx.x * CB;
  const float2* pin = P + (uint64_t)b * ln.in_bstride;
#pragma unroll
  for (int it0 = 0; it0 < CB * R2; it0 += kT) {
    const int it = it0 + threadIdx.x;
    if ((CB * R2) % kT != 0 && it >= CB * R2) break;
    const int col = it % CB, m2 = it / CB;
    const int cg = c0 + col;
    float2 v[R1];
#pragma unroll
    for (int m1 = 0; m1 < R1; ++m1) {
      const int i = R2 * m1 + m2 - ln.off;
      v[m1] = (cg < ln.ncols && i >= 0 && i < ln.nio) ? pin[(uint64_t)i * ln.rstride + cg] : make_float2(0.f, 0.f);
    }
    dft<R1>(v, false);
    float2* d = sh + m2 * CB + col;
    d[0] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1) d[k1 * R2 * CB] = twiddle(v[k1], tw[k1 * R2 + m2], false);
  }
  __syncthreads();
  float2* pout = out + (uint64_t)b * ln.out_bstride;
#pragma unroll
  for (int it0 = 0; it0 < CB * R1; it0 += kT) {
    const int it = it0 + threadIdx.x;
    if ((CB * R1) % kT != 0 && it >= CB * R1) break;
    const int col = it % CB, k1 = it / CB;
    const int cg = c0 + col;
    float2 u[R2];
    const float2* s = sh + k1 * R2 * CB + col;
#pragma unroll
    for (int m2 = 0; m2 < R2; ++m2) u[m2] = s[m2 * CB];
    dft<R2>(u, false);
    if (cg < ln.ncols) {
      float2* o = pout + (uint64_t)k1 * ln.rstride + cg;
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) o[(uint64_t)R1 * k2 * ln.rstride] = u[k2];
    }
  }
}

// Inverse strided lines: per column, all n rows, inverse FFT along the line,
// keep the nio rows at off + i -> row i of the output.  Every input cell is
// read exactly once; with CLEAR it is zeroed after that read (through inw,
// the same grids), which leaves them zero for the next adjoint spread;
// without it the input is read-only (in).
template <int LOGN, bool CLEAR>
__global__ void __launch_bounds__(kT) k_fft_inv_cols(Lines ln, const float2* __restrict__ in, float2* inw,
                                                     const float2* __restrict__ tw, float2* __restrict__ Q) {
  pdl_wait();
  using CG = ColGeo<LOGN>;
  constexpr int R1 = CG::R1, R2 = CG::R2, CB = CG::CB;
  extern __shared__ float2 sh[];
  const int b = blockIdx.y, c0 = blockIdx.x * CB;
#pragma unroll
  for (int it0 = 0; it0 < CB * R2; it0 += kT) {
    const int it = it0 + threadIdx.x;
    if ((CB * R2) % kT != 0 && it >= CB * R2) break;
    const int col = it % CB, m2 = it / CB;
    const int cg = c0 + col;
    const uint64_t o = (uint64_t)b * ln.in_bstride + (uint64_t)m2 * ln.rstride + cg;
    float2 v[R1];
    if constexpr (CLEAR) {
#pragma unroll
      for (int m1 = 0; m1 < R1; ++m1)
        v[m1] = (cg < ln.ncols) ? inw[o + (uint64_t)R2 * m1 * ln.rstride] : make_float2(0.f, 0.f);
    } else {
#pragma unroll
      for (int m1 = 0; m1 < R1; ++m1)
        v[m1] = (cg < ln.ncols) ? in[o + (uint64_t)R2 * m1 * ln.rstride] : make_float2(0.f, 0.f);
    }
    dft<R1>(v, true);
    float2* d = sh + m2 * CB + col;
    d[0] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1) d[k1 * R2 * CB] = twiddle(v[k1], tw[k1 * R2 + m2], true);
    if constexpr (CLEAR) {
      if (cg < ln.ncols) {
#pragma unroll
        for (int m1 = 0; m1 < R1; ++m1) inw[o + (uint64_t)R2 * m1 * ln.rstride] = make_float2(0.f, 0.f);
      }
    }
  }
  __syncthreads();
  float2* pout = Q + (uint64_t)b * ln.out_bstride;
#pragma unroll
  for (int it0 = 0; it0 < CB * R1; it0 += kT) {
    const int it = it0 + threadIdx.x;
    if ((CB * R1) % kT != 0 && it >= CB * R1) break;
    const int col = it % CB, k1 = it / CB;
    const int cg = c0 + col;
    float2 u[R2];
    const float2* s = sh + k1 * R2 * CB + col;
#pragma unroll
    for (int m2 = 0; m2 < R2; ++m2) u[m2] = s[m2 * CB];
    dft<R2>(u, true);
    if (cg >= ln.ncols) continue;
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      const int i = k1 + R1 * k2 - ln.off;
      if (i >= 0 && i < ln.nio) pout[(uint64_t)i * ln.rstride + cg] = u[k2];
    }
  }
}

// Last inverse pass: cropped lines (ix, iz) of grid b, inverse FFT along y,
// keep gy = crop + iy and apply the post-kernel weights of grid b = (coil c,
// segment l) -> Rimg[b][p].
template <int LOGN>
__global__ void __launch_bounds__(kT) k_fft_inv_rows(NufftGeom g, int L, const float2* __restrict__ Q,
                                                     const float2* __restrict__ S, int c0,
                                                     const float2* __restrict__ E, const float2* __restrict__ WoH,
                                                     const float* __restrict__ deapf, const float2* __restrict__ tw,
                                                     float2* __restrict__ Rimg) {
  pdl_wait();
  using RG = RowGeo<LOGN>;
  constexpr int R1 = RG::R1, R2 = RG::R2, n = RG::n, RB = RG::RB, S2 = RG::S2, RS = RG::RS;
  extern __shared__ float2 sh[];
  constexpr int Nn = n / 2;
  const int crop = g.crop_off[1];
  const int nrows = g.Nx * g.Nz;
  const uint64_t N = g.nimg();
  const int b = blockIdx.y, c = b / L, l = b - c * L;
  const int r0 = blockIdx.x * RB;
  {
    const int m2 = threadIdx.x % R2, r = threadIdx.x / R2;
    const int rg = r0 + r;
    float2 v[R1];
    const float2* s = Q + ((uint64_t)b * nrows + rg) * n + m2;
#pragma unroll
    for (int m1 = 0; m1 < R1; ++m1) v[m1] = (rg < nrows) ? s[R2 * m1] : make_float2(0.f, 0.f);
    dft<R1>(v, true);
    float2* d = sh + r * RS + m2;
    d[0] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < R1; ++k1) d[k1 * S2] = twiddle(v[k1], tw[k1 * R2 + m2], true);
  }
  __syncthreads();
#pragma unroll
  for (int it0 = 0; it0 < RB * R1; it0 += kT) {
    const int it = it0 + threadIdx.x;
    if ((RB * R1) % kT != 0 && it >= RB * R1) break;
    const int k1 = it % R1, r = it / R1;
    const int rg = r0 + r;
    float2 u[R2];
    const float2* s = sh + r * RS + k1 * S2;
#pragma unroll
    for (int m2 = 0; m2 < R2; ++m2) u[m2] = s[m2];
    dft<R2>(u, true);
    if (rg >= nrows) continue;
    const int ix = rg % g.Nx, iz = rg / g.Nx;
    const int pxz = ix + g.crop_off[0] + iz + g.crop_off[2];
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      const int iy = k1 + R1 * k2 - crop;
      if (iy < 0 || iy >= Nn) continue;
      const uint64_t p = (uint64_t)iy + (uint64_t)Nn * ((uint64_t)ix + (uint64_t)g.Nx * iz);
      float2 v = u[k2];
      const float f = parity2(pxz, iy + crop) ? -deapf[p] : deapf[p];
      v = make_float2(v.x * f, v.y * f);
      if (WoH) v = cmul(v, WoH[(uint64_t)l * N + p]);
      if (S) {
        const float2 sv = S[(uint64_t)(c0 + c) * N + p];
        v = E ? cmul(cmul(cconj(sv), cconj(E[p])), v) : cmul(v, cconj(sv));
      }
      Rimg[(uint64_t)b * N + p] = v;
    }
  }
}

// x[p] (+)= sum over the batch's grids of Rimg[b][p]: 8 lanes per pixel, lane
// k takes grids k, k+8, ..., added by a fixed xor butterfly.
__global__ void k_sum_images(uint64_t N, int B, const float2* __restrict__ Rimg, int accumulate,
                             float2* __restrict__ x) {
  pdl_wait();
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
pg_status rows_fwd(const NufftGeom& g, int B, int L, const float2* x, const float2* S, int c0, const float2* E,
                   const float2* Wo, const float* deapf, const float2* tw, float2* P, cudaStream_t s) {
  using RG = RowGeo<LOGN>;
  PG_CUDA(cudaFuncSetAttribute(k_fft_fwd_rows<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RG::smem));
  PG_LAUNCH_PDL(k_fft_fwd_rows<LOGN>, dim3(ceil_div((uint64_t)g.Nx * g.Nz, RG::RB), B), kT, RG::smem, s, g, L, x, S, c0,
            E, Wo, deapf, tw, P);
  return PG_OK;
}

template <int LOGN>
pg_status rows_inv(const NufftGeom& g, int B, int L, const float2* Q, const float2* S, int c0, const float2* E,
                   const float2* WoH, const float* deapf, const float2* tw, float2* Rimg, cudaStream_t s) {
  using RG = RowGeo<LOGN>;
  PG_CUDA(cudaFuncSetAttribute(k_fft_inv_rows<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RG::smem));
  PG_LAUNCH_PDL(k_fft_inv_rows<LOGN>, dim3(ceil_div((uint64_t)g.Nx * g.Nz, RG::RB), B), kT, RG::smem, s, g, L, Q, S, c0,
            E, WoH, deapf, tw, Rimg);
  return PG_OK;
}

template <int LOGN>
pg_status cols_fwd(const Lines& ln, int B, const float2* P, const float2* tw, float2* out, cudaStream_t s) {
  using CG = ColGeo<LOGN>;
  PG_CUDA(cudaFuncSetAttribute(k_fft_fwd_cols<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CG::smem));
  PG_LAUNCH_PDL(k_fft_fwd_cols<LOGN>, dim3(ceil_div(ln.ncols, CG::CB), B), kT, CG::smem, s, ln, P, tw, out);
  return PG_OK;
}

template <int LOGN>
pg_status cols_inv(const Lines& ln, int B, float2* in, int clear, const float2* tw, float2* Q, cudaStream_t s) {
  using CG = ColGeo<LOGN>;
  if (clear) {
    PG_CUDA(cudaFuncSetAttribute(k_fft_inv_cols<LOGN, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)CG::smem));
    PG_LAUNCH_PDL((k_fft_inv_cols<LOGN, true>), dim3(ceil_div(ln.ncols, CG::CB), B), kT, CG::smem, s, ln, in, in, tw, Q);
  } else {
    PG_CUDA(cudaFuncSetAttribute(k_fft_inv_cols<LOGN, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)CG::smem));
    PG_LAUNCH_PDL((k_fft_inv_cols<LOGN, false>), dim3(ceil_div(ln.ncols, CG::CB), B), kT, CG::smem, s, ln, in, nullptr,
              tw, Q);
  }
  return PG_OK;
}

#define PG_FFT_DISPATCH(lg, fn, ...)                                           \
  switch (lg) {                                                                \
    case 4: return fn<4>(__VA_ARGS__);                                         \
    case 5: return fn<5>(__VA_ARGS__);                                         \
    case 6: return fn<6>(__VA_ARGS__);                                         \
    case 7: return fn<7>(__VA_ARGS__);                                         \
    case 8: return fn<8>(__VA_ARGS__);                                         \
    case 9: return fn<9>(__VA_ARGS__);                                         \
    case 10: return fn<10>(__VA_ARGS__);                                       \
    default: return set_error(PG_INVALID_ARG, "fft passes: unsupported length 2^%d", lg); \
  }

pg_status d_rows_fwd(int lg, const NufftGeom& g, int B, int L, const float2* x, const float2* S, int c0,
                     const float2* E, const float2* Wo, const float* deapf, const float2* tw, float2* P,
                     cudaStream_t s) {
  PG_FFT_DISPATCH(lg, rows_fwd, g, B, L, x, S, c0, E, Wo, deapf, tw, P, s)
}
pg_status d_rows_inv(int lg, const NufftGeom& g, int B, int L, const float2* Q, const float2* S, int c0,
                     const float2* E, const float2* WoH, const float* deapf, const float2* tw, float2* Rimg,
                     cudaStream_t s) {
  PG_FFT_DISPATCH(lg, rows_inv, g, B, L, Q, S, c0, E, WoH, deapf, tw, Rimg, s)
}
pg_status d_cols_fwd(int lg, const Lines& ln, int B, const float2* P, const float2* tw, float2* out, cudaStream_t s) {
  PG_FFT_DISPATCH(lg, cols_fwd, ln, B, P, tw, out, s)
}
pg_status d_cols_inv(int lg, const Lines& ln, int B, float2* in, int clear, const float2* tw, float2* Q,
                     cudaStream_t s) {
  PG_FFT_DISPATCH(lg, cols_inv, ln, B, in, clear, tw, Q, s)
}

// ---------------------------------------------------------------------------
// Fused 2-D passes for 256 x 256 grids: one thread-block cluster of CL = 4
// CTAs per grid.
//   forward  CTA r transforms image rows [32r, 32r+32) along y (the F1
//            arithmetic, pre weights included) into its own shared memory;
//            after a cluster barrier it transforms grid columns [64r, 64r+64)
//            along x, reading the 128 nonzero rows from the four CTAs'
//            shared memory (distributed shared memory), and stores the full
//            columns (the F2 arithmetic).
//   adjoint  CTA r inverse-transforms grid columns [64r, 64r+64) along x and
//            keeps the 128 cropped rows in its shared memory (A1); after a
//            cluster barrier it inverse-transforms cropped rows [32r, 32r+32)
//            along y, reading the 256 columns from the four CTAs, and applies
//            the post weights (A2).
// The transforms are the separate passes' code in the same order, so the
// results are the same floats; the half-transformed grid never leaves the
// SMs and one launch replaces two.  Every thread of every CTA reaches both
// cluster barriers (no early exits); the second keeps each CTA's rows alive
// until the other CTAs have read them.
// ---------------------------------------------------------------------------
namespace fused {
constexpr int n = 256, Nn = 128, R = 16;   // n = R * R (Split<8>)
constexpr int CL = 4;                      // CTAs per grid
constexpr int kTF = 512;                   // threads per CTA
constexpr int RPC = Nn / CL;               // image rows per CTA
constexpr int CPC = n / CL;                // grid columns per CTA
constexpr int S2 = RowGeo<8>::S2, RS = RowGeo<8>::RS;
constexpr int kHeld = RPC * n;             // rows (forward) or cropped columns (adjoint) held for the cluster
constexpr int kWork = (n * CPC > RPC * RS) ? n * CPC : RPC * RS;
constexpr size_t smem = (size_t)(kHeld + kWork) * sizeof(float2);
static_assert(RowGeo<8>::R1 == R && RowGeo<8>::R2 == R, "four-step split of 256");
static_assert(kTF == RPC * R && CPC * R % kTF == 0, "thread mapping");
static_assert(Nn * CPC == kHeld, "held block sizes");
}  // namespace fused

__global__ void __launch_bounds__(fused::kTF, 1)
    k_fft2_fwd_fused(NufftGeom g, int L, const float2* __restrict__ x, const float2* __restrict__ S, int c0,
                     const float2* __restrict__ E, const float2* __restrict__ Wo, const float* __restrict__ deapf,
                     const float2* __restrict__ tw, float2* __restrict__ grids) {
  pdl_wait();
  using namespace fused;
  extern __shared__ float2 sh[];
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  float2* P = sh;               // [row][gy], this CTA's 32 image rows after the y transform
  float2* W = sh + kHeld;       // work area
  const int pad = g.pad_off[1];
  const uint64_t N = g.nimg();
  const int b = blockIdx.y, c = b / L, l = b - c * L;
  {  // y transform, pass 1: one (row, m2) per thread
    const int m2 = threadIdx.x % R, rl = threadIdx.x / R;
    const int ix = r * RPC + rl;
    const int px = ix + g.pad_off[0];
    float2 v[R];
#pragma unroll
    for (int m1 = 0; m1 < R; ++m1) {
      const int gy = R * m1 + m2;
      const int iy = gy - pad;
      float2 u = make_float2(0.f, 0.f);
      if (iy >= 0 && iy < Nn) {
        const uint64_t p = (uint64_t)iy + (uint64_t)Nn * ix;
        u = x[p];
        if (S) {
          const float2 sv = S[(uint64_t)(c0 + c) * N + p];
          u = E ? cmul(u, cmul(sv, E[p])) : cmul(sv, u);
        }
        if (Wo) u = cmul(Wo[(uint64_t)l * N + p], u);
        const float f = parity2(px, gy) ? -deapf[p] : deapf[p];
        u = make_float2(u.x * f, u.y * f);
      }
      v[m1] = u;
    }
    dft<R>(v, false);
    float2* d = W + rl * RS + m2;
    d[0] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) d[k1 * S2] = twiddle(v[k1], tw[k1 * R + m2], false);
  }
  __syncthreads();
  {  // y transform, pass 2: one (row, k1) per thread
    const int k1 = threadIdx.x % R, rl = threadIdx.x / R;
    float2 u[R];
    const float2* s = W + rl * RS + k1 * S2;
#pragma unroll
    for (int m2 = 0; m2 < R; ++m2) u[m2] = s[m2];
    dft<R>(u, false);
    float2* o = P + rl * n + k1;
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2) o[R * k2] = u[k2];
  }
  cluster.sync();
  const int padx = g.pad_off[0];
  for (int it = threadIdx.x; it < CPC * R; it += kTF) {   // x transform, pass 1: (column, m2)
    const int col = it % CPC, m2 = it / CPC;
    const int gy = r * CPC + col;
    float2 v[R];
#pragma unroll
    for (int m1 = 0; m1 < R; ++m1) {
      const int ix = R * m1 + m2 - padx;
      v[m1] = (ix >= 0 && ix < Nn) ? *cluster.map_shared_rank(P + (ix % RPC) * n + gy, ix / RPC)
                                   : make_float2(0.f, 0.f);
    }
    dft<R>(v, false);
    float2* d = W + m2 * CPC + col;
    d[0] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) d[k1 * R * CPC] = twiddle(v[k1], tw[k1 * R + m2], false);
  }
  __syncthreads();
  float2* out = grids + (uint64_t)b * n * n;
  for (int it = threadIdx.x; it < CPC * R; it += kTF) {   // x transform, pass 2: (column, k1)
    const int col = it % CPC, k1 = it / CPC;
    float2 u[R];
    const float2* s = W + k1 * R * CPC + col;
#pragma unroll
    for (int m2 = 0; m2 < R; ++m2) u[m2] = s[m2 * CPC];
    dft<R>(u, false);
    float2* o = out + (uint64_t)k1 * n + r * CPC + col;
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2) o[(uint64_t)R * k2 * n] = u[k2];
  }
  cluster.sync();
}

template <bool CLEAR>
__global__ void __launch_bounds__(fused::kTF, 1)
    k_fft2_adj_fused(NufftGeom g, int L, const float2* __restrict__ grids, float2* gridsw,
                     const float2* __restrict__ S, int c0,
                     const float2* __restrict__ E, const float2* __restrict__ WoH, const float* __restrict__ deapf,
                     const float2* __restrict__ tw, float2* __restrict__ Rimg) {
  pdl_wait();
  using namespace fused;
  extern __shared__ float2 sh[];
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  float2* Q = sh;               // [cropped row][column], this CTA's 64 columns after the x transform
  float2* W = sh + kHeld;
  const int crop0 = g.crop_off[0], crop1 = g.crop_off[1];
  const uint64_t N = g.nimg();
  const int b = blockIdx.y, c = b / L, l = b - c * L;
  for (int it = threadIdx.x; it < CPC * R; it += kTF) {   // x transform, pass 1: (column, m2)
    const int col = it % CPC, m2 = it / CPC;
    const uint64_t o = (uint64_t)b * n * n + (uint64_t)m2 * n + r * CPC + col;
    float2 v[R];
    if constexpr (CLEAR) {
#pragma unroll
      for (int m1 = 0; m1 < R; ++m1) v[m1] = gridsw[o + (uint64_t)R * m1 * n];
    } else {
#pragma unroll
      for (int m1 = 0; m1 < R; ++m1) v[m1] = grids[o + (uint64_t)R * m1 * n];
    }
    dft<R>(v, true);
    float2* d = W + m2 * CPC + col;
    d[0] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) d[k1 * R * CPC] = twiddle(v[k1], tw[k1 * R + m2], true);
    if constexpr (CLEAR) {   // every grid cell is read once, here: zero it for the next adjoint spread
#pragma unroll
      for (int m1 = 0; m1 < R; ++m1) gridsw[o + (uint64_t)R * m1 * n] = make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < CPC * R; it += kTF) {   // x transform, pass 2: keep the cropped rows
    const int col = it % CPC, k1 = it / CPC;
    float2 u[R];
    const float2* s = W + k1 * R * CPC + col;
#pragma unroll
    for (int m2 = 0; m2 < R; ++m2) u[m2] = s[m2 * CPC];
    dft<R>(u, true);
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2) {
      const int i = k1 + R * k2 - crop0;
      if (i >= 0 && i < Nn) Q[i * CPC + col] = u[k2];
    }
  }
  cluster.sync();
  {  // y transform, pass 1: one (cropped row, m2) per thread, columns from the four CTAs
    const int m2 = threadIdx.x % R, rl = threadIdx.x / R;
    const int ix = r * RPC + rl;
    float2 v[R];
#pragma unroll
    for (int m1 = 0; m1 < R; ++m1) {
      const int gy = R * m1 + m2;
      v[m1] = *cluster.map_shared_rank(Q + ix * CPC + gy % CPC, gy / CPC);
    }
    dft<R>(v, true);
    float2* d = W + rl * RS + m2;
    d[0] = v[0];
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) d[k1 * S2] = twiddle(v[k1], tw[k1 * R + m2], true);
  }
  __syncthreads();
  {  // y transform, pass 2: keep the cropped columns, post weights
    const int k1 = threadIdx.x % R, rl = threadIdx.x / R;
    const int ix = r * RPC + rl;
    float2 u[R];
    const float2* s = W + rl * RS + k1 * S2;
#pragma unroll
    for (int m2 = 0; m2 < R; ++m2) u[m2] = s[m2];
    dft<R>(u, true);
    const int px = ix + crop0;
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2) {
      const int iy = k1 + R * k2 - crop1;
      if (iy < 0 || iy >= Nn) continue;
      const uint64_t p = (uint64_t)iy + (uint64_t)Nn * ix;
      float2 v = u[k2];
      const float f = parity2(px, iy + crop1) ? -deapf[p] : deapf[p];
      v = make_float2(v.x * f, v.y * f);
      if (WoH) v = cmul(v, WoH[(uint64_t)l * N + p]);
      if (S) {
        const float2 sv = S[(uint64_t)(c0 + c) * N + p];
        v = E ? cmul(cmul(cconj(sv), cconj(E[p])), v) : cmul(v, cconj(sv));
      }
      Rimg[(uint64_t)b * N + p] = v;
    }
  }
  cluster.sync();
}

template <typename Kern, typename... Args>
pg_status launch_fused(Kern kern, int B, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(fused::CL, (unsigned)B, 1);
  cfg.blockDim = dim3(fused::kTF, 1, 1);
  cfg.dynamicSmemBytes = fused::smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = fused::CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;   // the kernels call pdl_wait()
  attr[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  PG_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
  count_launch();
  return PG_OK;
}

// The fused passes run where a cluster of four 192 KB CTAs can be resident
// (queried once per process; plan creation may run on several threads).
bool query_fused() {
  if (cudaFuncSetAttribute(k_fft2_fwd_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused::smem) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_fft2_adj_fused<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused::smem) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_fft2_adj_fused<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused::smem) !=
          cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(fused::CL, 1, 1);
  cfg.blockDim = dim3(fused::kTF, 1, 1);
  cfg.dynamicSmemBytes = fused::smem;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = fused::CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;   // the kernels call pdl_wait()
  attr[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  int nf = 0, na = 0;
  if (cudaOccupancyMaxActiveClusters(&nf, k_fft2_fwd_fused, &cfg) != cudaSuccess ||
      cudaOccupancyMaxActiveClusters(&na, k_fft2_adj_fused<true>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return nf >= 1 && na >= 1;
}

bool fused_available() {
  static const bool ok = query_fused();   // thread-safe one-time initialisation
  return ok;
}

// PG_FFT_FUSED=0 (read at each call) keeps the separate passes.
bool use_fused(const NufftGeom& g) {
  const char* e = getenv("PG_FFT_FUSED");
  if (e && e[0] == '0') return false;
  return g.dim == 2 && g.Gx == fused::n && g.Gy == fused::n && g.Nx == fused::Nn && g.Ny == fused::Nn &&
         fused_available();
}

int log2_exact(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return ((1 << l) == v) ? l : -1;
}

// R2 of the factorisation n = R1 * R2 (Split above).
int split_r2(int n) { return n >= 1024 ? 32 : n <= 64 ? 4 : n / 16; }

void twiddle_table(int n, std::vector<float2>* h) {
  const int R2 = split_r2(n), R1 = n / R2;
  const double two_pi = 6.283185307179586476925286766559;
  for (int k1 = 0; k1 < R1; ++k1)
    for (int m2 = 0; m2 < R2; ++m2) {
      const double a = -two_pi * (double)(k1 * m2) / (double)n;
      h->push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
    }
}

}  // namespace

bool fftpass_supported(const NufftGeom& g) {
  if (g.Gx != g.Gy || g.Gx != 2 * g.Nx || g.Ny != g.Nx) return false;
  const int l = log2_exact(g.Gx);
  if (l < 4 || l > 10) return false;
  if (g.dim == 2) return true;
  const int lz = log2_exact(g.Gz);
  return g.Gz == 2 * g.Nz && lz >= 4 && lz <= 10;
}

uint64_t fftpass_scratch(const NufftGeom& g, int B) {
  // 2-D: Nx rows of Gy per grid.  3-D: Nz*Nx rows of Gy, then Nz slabs of Gx*Gy.
  const uint64_t rows = (uint64_t)g.Nx * g.Nz * g.Gy;
  return (uint64_t)B * (g.dim == 2 ? rows : rows + (uint64_t)g.Nz * g.Gx * g.Gy);
}

pg_status fftpass_twiddles(const NufftGeom& g, DevBuf<float2>* tw, cudaStream_t s) {
  std::vector<float2> h;
  twiddle_table(g.Gx, &h);
  if (g.dim == 3) twiddle_table(g.Gz, &h);   // the z table follows the in-plane one
  else (void)fused_available();              // occupancy query outside any stream capture
  return tw->upload(h.data(), h.size(), s);
}

pg_status fftpass_forward(const NufftGeom& g, int B, int L, const float2* x, const float2* S, int c0,
                          const float2* E, const float2* Wo, const float* deapf, const float2* tw, float2* P,
                          float2* grids, cudaStream_t s) {
  if (B > kMaxGridY) return set_error(PG_INVALID_ARG, "fft passes: batch of %d grids", B);
  if (use_fused(g)) return launch_fused(k_fft2_fwd_fused, B, s, g, L, x, S, c0, E, Wo, deapf, tw, grids);
  const int lg = log2_exact(g.Gx);
  const uint64_t plane = (uint64_t)g.Gx * g.Gy;
  PG_TRY(d_rows_fwd(lg, g, B, L, x, S, c0, E, Wo, deapf, tw, P, s));
  if (g.dim == 2) {
    const Lines ln{(uint64_t)g.Nx * g.Gy, plane, (uint64_t)g.Gy, g.Gy, g.Nx, g.pad_off[0]};
    return d_cols_fwd(lg, ln, B, P, tw, grids, s);
  }
  // x lines per nonzero z-slab, then z lines over every (x, y) column
  float2* P2 = P + (uint64_t)B * g.Nz * g.Nx * g.Gy;
  const Lines lx{(uint64_t)g.Nx * g.Gy, plane, (uint64_t)g.Gy, g.Gy, g.Nx, g.pad_off[0]};
  const int slabs = B * g.Nz;
  for (int s0 = 0; s0 < slabs; s0 += kMaxGridY)
    PG_TRY(d_cols_fwd(lg, lx, std::min(kMaxGridY, slabs - s0), P + s0 * lx.in_bstride, tw,
                      P2 + s0 * lx.out_bstride, s));
  const Lines lz{(uint64_t)g.Nz * plane, g.ngrid(), plane, (int)plane, g.Nz, g.pad_off[2]};
  return d_cols_fwd(log2_exact(g.Gz), lz, B, P2, tw + g.Gx, grids, s);
}

pg_status fftpass_adjoint(const NufftGeom& g, int B, int L, float2* grids, int clear, const float2* S, int c0,
                          const float2* E, const float2* WoH, const float* deapf, const float2* tw, float2* Q,
                          float2* Rimg, int accumulate, float2* x, cudaStream_t s) {
  if (B > kMaxGridY) return set_error(PG_INVALID_ARG, "fft passes: batch of %d grids", B);
  const int lg = log2_exact(g.Gx);
  const uint64_t plane = (uint64_t)g.Gx * g.Gy;
  float2* Qr = Q;   // the rows the last pass reads
  if (use_fused(g)) {
    if (clear)
      PG_TRY(launch_fused(k_fft2_adj_fused<true>, B, s, g, L, (const float2*)grids, grids, S, c0, E, WoH, deapf, tw,
                          Rimg));
    else
      PG_TRY(launch_fused(k_fft2_adj_fused<false>, B, s, g, L, (const float2*)grids, (float2*)nullptr, S, c0, E,
                          WoH, deapf, tw, Rimg));
    const uint64_t N = g.nimg();
    PG_LAUNCH_PDL(k_sum_images, ceil_div(N * 8, 256), 256, 0, s, N, B, Rimg, accumulate, x);
    return PG_OK;
  }
  if (g.dim == 2) {
    const Lines ln{plane, (uint64_t)g.Nx * g.Gy, (uint64_t)g.Gy, g.Gy, g.Nx, g.crop_off[0]};
    PG_TRY(d_cols_inv(lg, ln, B, grids, clear, tw, Q, s));
  } else {
    // z lines keeping the Nz cropped slabs, then x lines per slab keeping Nx rows
    float2* Q1 = Q + (uint64_t)B * g.Nz * g.Nx * g.Gy;
    const Lines lz{g.ngrid(), (uint64_t)g.Nz * plane, plane, (int)plane, g.Nz, g.crop_off[2]};
    PG_TRY(d_cols_inv(log2_exact(g.Gz), lz, B, grids, clear, tw + g.Gx, Q1, s));
    const Lines lx{plane, (uint64_t)g.Nx * g.Gy, (uint64_t)g.Gy, g.Gy, g.Nx, g.crop_off[0]};
    const int slabs = B * g.Nz;
    for (int s0 = 0; s0 < slabs; s0 += kMaxGridY)
      PG_TRY(d_cols_inv(lg, lx, std::min(kMaxGridY, slabs - s0), Q1 + s0 * lx.in_bstride, 0, tw,
                        Q + s0 * lx.out_bstride, s));
  }
  PG_TRY(d_rows_inv(lg, g, B, L, Qr, S, c0, E, WoH, deapf, tw, Rimg, s));
  const uint64_t N = g.nimg();
  PG_LAUNCH_PDL(k_sum_images, ceil_div(N * 8, 256), 256, 0, s, N, B, Rimg, accumulate, x);
  return PG_OK;
}

}  // namespace pg
