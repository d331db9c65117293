// Gridding NUFFT for sm_100a.
//
// Reference semantics (paths relative to PowerGrid/):
//   forward  computeFd_CPU_Grid  gridding.cpp:584-727
//            deapodize -> zero_pad -> fftshift -> FFT(-1) -> ifftshift -> interpolate
//   adjoint  computeFH_CPU_Grid  gridding.cpp:418-581
//            spread -> ifftshift -> FFT(+1) -> fftshift -> crop -> deapodize
//   window   clamped [ceil(s-W*os/2), floor(s+W*os/2)], s = os*(k + N/2)   gridding.cpp:64-73
//   weight   nearest-lower LUT entry, 0 past the end                       gridding.cpp:78-84
// FFTs are unnormalised (gridding.cpp:540-549 left commented out).
//
// B200 design:
//   * every shift, pad and crop is index arithmetic inside the pre/post and
//     gridding kernels — no full-grid copy passes;
//   * deapodization, coil maps (SENSE), segment phases Wo/WoH
//     (TimeSegmentation) and shot phases (pcSenseTimeSeg) are fused into
//     the pre/post kernels, so one launch covers all coils x segments;
//   * the time-segment interpolator AA is applied inside the gridding pass:
//     each sample is read once and contributes to its K nonzero segments;
//   * samples are binned once per trajectory (stable counting sort by
//     (segment window, tile)); the adjoint spreads each bin into a padded
//     shared-memory tile and flushes the tile once, so global atomics are
//     per tile cell, not per tap;
//   * cuFFT runs only the oversampled FFT, batched over coils x segments.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "pg_nufft.cuh"
#include "pg_profile.cuh"

namespace pg {

// ---------------------------------------------------------------------------
// Host tables, with the operand types of the reference so the values agree.
// ---------------------------------------------------------------------------
namespace {

constexpr float kPiF = 3.1415926535897932384626433832795029f;  // PGIncludes.h:69

// I0 by the Abramowitz & Stegun 9.8.1/9.8.2 polynomials (griddingSupport.cpp:33-48).
float bessel_i0f(float x) {
  float ax = std::abs(x);
  float y, r;
  if (ax < 3.75) {
    y = x / 3.75;
    y = y * y;
    r = 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 +
        y * (0.2659732 + y * (0.360768e-1 + y * 0.45813e-2)))));
  } else {
    y = 3.75 / ax;
    r = (std::exp(ax) / std::sqrt(ax)) *
        (0.39894228 + y * (0.1328592e-1 + y * (0.225319e-2 + y * (-0.157565e-2 +
        y * (0.916281e-2 + y * (-0.2057706e-1 + y * (0.2635537e-1 +
        y * (-0.1647633e-1 + y * 0.392377e-2))))))));
  }
  return r;
}

// Reciprocal Kaiser-Bessel transform factor along one axis
// (griddingSupport.cpp:246-262 for 2-D; :327-348 for 3-D).
float deapod_factor(int i, int n, float kw, float beta, bool three_d) {
  float u;
  if (three_d)
    u = (float)((i) - ((float)n / 2.0)) / (float)n;
  else
    u = (float)(i - (n / 2)) / (float)n;
  float c = kPiF * kPiF * kw * kw * u * u - beta * beta;
  if (c >= 0) return std::sin(std::sqrt(c)) / std::sqrt(c);
  if (three_d) return (float)(std::sinh(std::sqrt(-1.0 * c)) / std::sqrt(-1.0 * c));
  return std::sinh(std::sqrt((float)-1.0 * c)) / std::sqrt((float)-1.0 * c);
}

}  // namespace

void kb_table(float gridos, std::vector<float>* lut, float* beta_out) {
  const float kw = 4.0f;  // Gnufft.cpp:84
  float beta = kPiF * std::sqrt((gridos - 0.5) * (gridos - 0.5) * (kw * kw * 4.0) / (gridos * gridos) - 0.8);
  const uint64_t n = (uint64_t)(10000 * kw);  // griddingSupport.cpp:61
  lut->resize(n);
  for (int k = 0; k < (int)n; ++k) {
    float v = static_cast<float>(k) / static_cast<float>(n);
    (*lut)[k] = bessel_i0f(beta * std::sqrt(1.0 - (v))) / kw;
  }
  *beta_out = beta;
}

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

// Window of one axis and its 8 tap weights.  Arithmetic is the reference's
// float sequence with no contraction, so the LUT entry chosen is identical.
// A window has 9 cells only when s is an integer, and then both end cells
// sit at distance W/2 and weigh 0; the nonzero taps therefore always fit in
// 8 consecutive cells starting at `st`.  Cells outside [lo, hi] weigh 0.
__device__ __forceinline__ int axis_taps(float k, int n_img, float os, float kw, const float* __restrict__ lut,
                                         int nlut, float* w) {
  const float s = __fmul_rn(os, __fadd_rn(k, __fdiv_rn((float)n_img, 2.0f)));
  const float half = __fdiv_rn(__fmul_rn(kw, os), 2.0f);
  const int lo = (int)fmaxf(0.0f, ceilf(__fsub_rn(s, half)));
  const int hi = (int)fminf(__fsub_rn(__fmul_rn(os, (float)n_img), 1.0f), floorf(__fadd_rn(s, half)));
  const int st = (hi - lo == 8) ? lo + 1 : lo;
  const float kw2 = __fmul_rn(kw, kw);
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int c = st + a;
    float wv = 0.0f;
    if (c >= lo && c <= hi) {
      const float dist = __fdiv_rn(fabsf(__fsub_rn(s, (float)c)), os);
      const int k0 = (int)__fmul_rn(__fdiv_rn(__fmul_rn(__fmul_rn(dist, dist), 4.0f), kw2), (float)nlut);
      wv = (k0 >= nlut || k0 < 0) ? 0.0f : lut[k0];
    }
    w[a] = wv;
  }
  return st;
}

__device__ __forceinline__ int wrap(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// Per-sample preparation (original order): tap starts, separable weights and bin key.
__global__ void k_prepare(NufftGeom g, uint64_t M, const float* __restrict__ kx, const float* __restrict__ ky,
                          const float* __restrict__ kz, const float* __restrict__ lut, TileShape t,
                          const int* __restrict__ l0, uint2* __restrict__ start, float* __restrict__ wxy,
                          float* __restrict__ wz, uint32_t* __restrict__ key) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  float w[8];
  const int sx = axis_taps(kx[i], g.Nx, g.os, g.kw, lut, g.nlut, w);
#pragma unroll
  for (int a = 0; a < 8; ++a) wxy[i * 16 + a] = w[a];
  const int sy = axis_taps(ky[i], g.Ny, g.os, g.kw, lut, g.nlut, w);
#pragma unroll
  for (int a = 0; a < 8; ++a) wxy[i * 16 + 8 + a] = w[a];
  int sz = 0;
  if (g.dim == 3) {
    sz = axis_taps(kz[i], g.Nz, g.os, g.kw, lut, g.nlut, w);
#pragma unroll
    for (int a = 0; a < 8; ++a) wz[i * 8 + a] = w[a];
  }
  start[i] = make_uint2((uint32_t)sx | ((uint32_t)sy << 16), (uint32_t)sz);
  const int tx = sx / t.TX, ty = sy / t.TY, tz = sz / t.TZ;
  const int l = l0 ? l0[i] : 0;
  key[i] = (uint32_t)((((uint64_t)l * t.ntz + tz) * t.ntx + tx) * t.nty + ty);
}

__global__ void k_permute(uint64_t M, int dim, int K, const uint32_t* __restrict__ perm,
                          const uint2* __restrict__ start_in, const float* __restrict__ wxy_in,
                          const float* __restrict__ wz_in, uint2* __restrict__ start_out,
                          float* __restrict__ wxy_out, float* __restrict__ wz_out) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  const uint32_t i = perm[j];
  start_out[j] = start_in[i];
  const float4* src = reinterpret_cast<const float4*>(wxy_in + (uint64_t)i * 16);
  float4* dst = reinterpret_cast<float4*>(wxy_out + j * 16);
#pragma unroll
  for (int a = 0; a < 4; ++a) dst[a] = src[a];
  if (dim == 3) {
    const float4* s2 = reinterpret_cast<const float4*>(wz_in + (uint64_t)i * 8);
    float4* d2 = reinterpret_cast<float4*>(wz_out + j * 8);
    d2[0] = s2[0];
    d2[1] = s2[1];
  }
}

// ---------------------------------------------------------------------------
// Forward: pre-kernel (deapodize + maps + phases + zero-pad + fftshift)
// ---------------------------------------------------------------------------
__global__ void k_pre(NufftGeom g, int L, const float2* __restrict__ x, const float2* __restrict__ S, int c0,
                      const float2* __restrict__ E, const float2* __restrict__ Wo, const float* __restrict__ deap,
                      float scale, float2* __restrict__ grids) {
  const uint64_t G = g.ngrid();
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= G) return;
  const int b = blockIdx.y;           // grid within the batch
  const int cl = b / L, l = b % L;
  const int fy = (int)(q % g.Gy);
  const int fx = (int)((q / g.Gy) % g.Gx);
  const int fz = (int)(q / ((uint64_t)g.Gy * g.Gx));
  const int iy = wrap(fy - g.fs[1], g.Gy) - g.pad_off[1];
  const int ix = wrap(fx - g.fs[0], g.Gx) - g.pad_off[0];
  const int iz = (g.dim == 3) ? wrap(fz - g.fs[2], g.Gz) - g.pad_off[2] : 0;
  float2 v = make_float2(0.f, 0.f);
  if (iy >= 0 && iy < g.Ny && ix >= 0 && ix < g.Nx && iz >= 0 && iz < g.Nz) {
    const uint64_t N = g.nimg();
    const uint64_t p = (uint64_t)iy + (uint64_t)g.Ny * ((uint64_t)ix + (uint64_t)g.Nx * iz);
    v = x[p];
    if (S) {
      const float2 s = S[(uint64_t)(c0 + cl) * N + p];
      v = E ? cmul(v, cmul(s, E[p])) : cmul(s, v);
    }
    if (Wo) v = cmul(Wo[(uint64_t)l * N + p], v);
    float k = deap[ix] * deap[g.Nx + iy];
    if (g.dim == 3) k = k * deap[g.Nx + g.Ny + iz];
    v = (k == k) ? make_float2(__fmul_rn(__fdiv_rn(v.x, k), scale), __fmul_rn(__fdiv_rn(v.y, k), scale))
                 : make_float2(0.f, 0.f);
  }
  grids[(uint64_t)b * G + q] = v;
}

// ---------------------------------------------------------------------------
// Forward: interpolation (gather) with ifftshift folded into the reads and
// the segment interpolator applied per sample.  One thread per sample.
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void __launch_bounds__(128) k_gather(NufftGeom g, uint64_t M, const uint2* __restrict__ start,
                                                const float* __restrict__ wxy, const float* __restrict__ wz,
                                                const uint32_t* __restrict__ perm, const int* __restrict__ l0,
                                                const float2* __restrict__ aa, int K, int L,
                                                const float2* __restrict__ grids, int Cb,
                                                float2* __restrict__ data, uint64_t dstride) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const uint2 st = start[i];
  const int sx = st.x & 0xffff, sy = st.x >> 16, sz = st.y;
  float wx[8], wy[8], wzz[8];
  {
    const float4* w4 = reinterpret_cast<const float4*>(wxy + i * 16);
    float4 a = w4[0], b = w4[1], c = w4[2], d = w4[3];
    wx[0] = a.x; wx[1] = a.y; wx[2] = a.z; wx[3] = a.w; wx[4] = b.x; wx[5] = b.y; wx[6] = b.z; wx[7] = b.w;
    wy[0] = c.x; wy[1] = c.y; wy[2] = c.z; wy[3] = c.w; wy[4] = d.x; wy[5] = d.y; wy[6] = d.z; wy[7] = d.w;
    if (DIM == 3) {
      const float4* z4 = reinterpret_cast<const float4*>(wz + i * 8);
      float4 e = z4[0], f = z4[1];
      wzz[0] = e.x; wzz[1] = e.y; wzz[2] = e.z; wzz[3] = e.w; wzz[4] = f.x; wzz[5] = f.y; wzz[6] = f.z; wzz[7] = f.w;
    }
  }
  int py[8], px[8], pz[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    py[a] = wrap(sy + a - g.ifs[1], g.Gy);
    px[a] = wrap(sx + a - g.ifs[0], g.Gx) * g.Gy;
    if (DIM == 3) pz[a] = wrap(sz + a - g.ifs[2], g.Gz) * g.Gx * g.Gy;
  }
  const uint64_t G = g.ngrid();
  const int lbase = l0 ? l0[i] : 0;
  const uint32_t orig = perm[i];
  for (int c = 0; c < Cb; ++c) {
    float2 out = make_float2(0.f, 0.f);
    for (int j = 0; j < K; ++j) {
      const float2* gr = grids + ((uint64_t)c * L + lbase + j) * G;
      float ar = 0.f, ai = 0.f;
      if (DIM == 2) {
#pragma unroll
        for (int a = 0; a < 8; ++a) {
          if (wx[a] == 0.f) continue;
          const float2* row = gr + px[a];
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            if (wy[b] == 0.f) continue;
            const float w = wx[a] * wy[b];
            const float2 v = __ldg(row + py[b]);
            ar = fmaf(w, v.x, ar);
            ai = fmaf(w, v.y, ai);
          }
        }
      } else {
        for (int e = 0; e < 8; ++e) {
          if (wzz[e] == 0.f) continue;
          const float2* pl = gr + pz[e];
#pragma unroll
          for (int a = 0; a < 8; ++a) {
            if (wx[a] == 0.f) continue;
            const float2* row = pl + px[a];
#pragma unroll
            for (int b = 0; b < 8; ++b) {
              if (wy[b] == 0.f) continue;
              const float w = wx[a] * wy[b] * wzz[e];
              const float2 v = __ldg(row + py[b]);
              ar = fmaf(w, v.x, ar);
              ai = fmaf(w, v.y, ai);
            }
          }
        }
      }
      const float2 acc = make_float2(ar, ai);
      out = aa ? cadd(out, cmul(acc, aa[i * K + j])) : acc;
    }
    data[(uint64_t)c * dstride + orig] = out;
  }
}

// ---------------------------------------------------------------------------
// Adjoint: spread one subproblem (a bin's samples, one segment window) into
// a padded shared-memory tile with shared atomics; flush each nonzero tile
// cell to the ifftshifted grid position with one vector atomic.
// Shared layout: [coil][segment][re|im][PZ][PX][PY], PY = 8 (mod 32) so a
// warp's 32 lanes (8 y-taps x 4 x-taps) hit 32 distinct banks.
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void __launch_bounds__(256) k_spread(NufftGeom g, TileShape t, const int4* __restrict__ sub,
                                                const uint2* __restrict__ start, const float* __restrict__ wxy,
                                                const float* __restrict__ wz, const uint32_t* __restrict__ perm,
                                                const float2* __restrict__ aa, int K, int L,
                                                const float2* __restrict__ data, uint64_t dstride, int Cb,
                                                int Cc, float2* __restrict__ grids) {
  extern __shared__ float sm[];
  const int4 sp = sub[blockIdx.x];
  const int cfirst = blockIdx.y * Cc;            // first coil (within batch) of this block
  const int ncl = min(Cc, Cb - cfirst);
  const int tile = sp.x, lseg = sp.y, first = sp.z, count = sp.w;
  const int ty = tile % t.nty;
  const int txz = tile / t.nty;
  const int tx = txz % t.ntx;
  const int tz = txz / t.ntx;
  const int x0 = tx * t.TX, y0 = ty * t.TY, z0 = tz * t.TZ;
  const int cells = t.PX * t.PY * t.PZ;
  const int nplanes = ncl * K * 2;
  for (int q = threadIdx.x; q < nplanes * cells; q += blockDim.x) sm[q] = 0.f;
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int dy = lane & 7, dx = lane >> 3;
  for (int s = first + warp; s < first + count; s += nw) {
    const uint2 st = start[s];
    const int ox = (int)(st.x & 0xffff) - x0, oy = (int)(st.x >> 16) - y0;
    const int oz = (DIM == 3) ? (int)st.y - z0 : 0;
    const float wyv = wxy[(uint64_t)s * 16 + 8 + dy];
    const float wx0 = wxy[(uint64_t)s * 16 + dx];
    const float wx1 = wxy[(uint64_t)s * 16 + dx + 4];
    const uint32_t orig = perm[s];
    const int a0 = (ox + dx) * t.PY + oy + dy;
    const int a1 = a0 + 4 * t.PY;
    for (int c = 0; c < ncl; ++c) {
      const float2 d = data[(uint64_t)(cfirst + c) * dstride + orig];
      for (int j = 0; j < K; ++j) {
        const float2 v = aa ? cmul(cconj(aa[(uint64_t)s * K + j]), d) : d;
        float* pr = sm + ((c * K + j) * 2) * cells;
        float* pi = pr + cells;
        if (DIM == 2) {
          const float w0 = wx0 * wyv, w1 = wx1 * wyv;
          if (w0 != 0.f) { atomicAdd(pr + a0, w0 * v.x); atomicAdd(pi + a0, w0 * v.y); }
          if (w1 != 0.f) { atomicAdd(pr + a1, w1 * v.x); atomicAdd(pi + a1, w1 * v.y); }
        } else {
          const int plane = t.PX * t.PY;
#pragma unroll 2
          for (int e = 0; e < 8; ++e) {
            const float wzv = wz[(uint64_t)s * 8 + e];
            if (wzv == 0.f) continue;
            const int zo = (oz + e) * plane;
            const float w0 = wx0 * wyv * wzv, w1 = wx1 * wyv * wzv;
            if (w0 != 0.f) { atomicAdd(pr + zo + a0, w0 * v.x); atomicAdd(pi + zo + a0, w0 * v.y); }
            if (w1 != 0.f) { atomicAdd(pr + zo + a1, w1 * v.x); atomicAdd(pi + zo + a1, w1 * v.y); }
          }
        }
      }
    }
  }
  __syncthreads();

  const uint64_t G = g.ngrid();
  for (int q = threadIdx.x; q < cells; q += blockDim.x) {
    const int pyy = q % t.PY;
    const int pxx = (q / t.PY) % t.PX;
    const int pzz = q / (t.PY * t.PX);
    const int gy = y0 + pyy, gx = x0 + pxx, gz = z0 + pzz;
    if (gy >= g.Gy || gx >= g.Gx || gz >= g.Gz) continue;
    const int sy = (gy + g.ifs[1]) % g.Gy;
    const int sx = (gx + g.ifs[0]) % g.Gx;
    const int sz = (DIM == 3) ? (gz + g.ifs[2]) % g.Gz : 0;
    const uint64_t idx = (uint64_t)sy + (uint64_t)g.Gy * ((uint64_t)sx + (uint64_t)g.Gx * sz);
    for (int c = 0; c < ncl; ++c)
      for (int j = 0; j < K; ++j) {
        const float* pr = sm + ((c * K + j) * 2) * cells;
        const float re = pr[q], im = pr[cells + q];
        if (re != 0.f || im != 0.f)
          atomicAdd(grids + ((uint64_t)(cfirst + c) * L + lseg + j) * G + idx, make_float2(re, im));
      }
  }
}

// ---------------------------------------------------------------------------
// Adjoint: post-kernel (fftshift + crop + deapodize + WoH + coil combine)
// ---------------------------------------------------------------------------
__global__ void k_post(NufftGeom g, int Cb, int L, const float2* __restrict__ grids, const float2* __restrict__ S,
                       int c0, const float2* __restrict__ E, const float2* __restrict__ WoH,
                       const float* __restrict__ deap, float scale, int accumulate, float2* __restrict__ x) {
  const uint64_t N = g.nimg();
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int iy = (int)(p % g.Ny);
  const int ix = (int)((p / g.Ny) % g.Nx);
  const int iz = (int)(p / ((uint64_t)g.Ny * g.Nx));
  const int gy = wrap(iy + g.crop_off[1] - g.fs[1], g.Gy);
  const int gx = wrap(ix + g.crop_off[0] - g.fs[0], g.Gx);
  const int gz = (g.dim == 3) ? wrap(iz + g.crop_off[2] - g.fs[2], g.Gz) : 0;
  const uint64_t q = (uint64_t)gy + (uint64_t)g.Gy * ((uint64_t)gx + (uint64_t)g.Gx * gz);
  const uint64_t G = g.ngrid();
  float k = deap[ix] * deap[g.Nx + iy];
  if (g.dim == 3) k = k * deap[g.Nx + g.Ny + iz];
  const bool ok = (k == k);
  float2 acc = accumulate ? x[p] : make_float2(0.f, 0.f);
  for (int c = 0; c < Cb; ++c) {
    float2 img = make_float2(0.f, 0.f);
    for (int l = 0; l < L; ++l) {
      float2 v = grids[((uint64_t)c * L + l) * G + q];
      v = ok ? make_float2(__fmul_rn(__fdiv_rn(v.x, k), scale), __fmul_rn(__fdiv_rn(v.y, k), scale))
             : make_float2(0.f, 0.f);
      if (WoH) v = cmul(v, WoH[(uint64_t)l * N + p]);
      img = (l == 0) ? v : cadd(img, v);
    }
    if (S) {
      const float2 s = S[(uint64_t)(c0 + c) * N + p];
      img = E ? cmul(cmul(cconj(s), cconj(E[p])), img) : cmul(img, cconj(s));
    }
    acc = cadd(acc, img);
  }
  x[p] = acc;
}

// ---------------------------------------------------------------------------
// Plan construction
// ---------------------------------------------------------------------------
NufftPlan::~NufftPlan() {
  for (auto& kv : ffts) cufftDestroy(kv.second);
}

static TileShape choose_tiles(const NufftGeom& g) {
  TileShape t{};
  if (g.dim == 2) {
    t.TX = 32; t.TY = 32; t.TZ = 1;
    t.PX = t.TX + 8; t.PY = t.TY + 8; t.PZ = 1;     // PY = 40 = 8 (mod 32)
  } else {
    t.TX = 8; t.TY = 8; t.TZ = 8;
    t.PX = 16; t.PY = 24; t.PZ = 16;                // PY = 24: 4 x-taps hit 4 distinct bank groups
  }
  t.ntx = (g.Gx + t.TX - 1) / t.TX;
  t.nty = (g.Gy + t.TY - 1) / t.TY;
  t.ntz = (g.Gz + t.TZ - 1) / t.TZ;
  return t;
}

pg_status nufft_plan_create(std::unique_ptr<NufftPlan>* out, uint64_t M, float gridos, int nx, int ny, int nz,
                            const float* kx, const float* ky, const float* kz, cudaStream_t s) {
  if (M == 0 || nx < 1 || ny < 1 || nz < 1) return set_error(PG_INVALID_ARG, "Gnufft: empty geometry");
  if (gridos != 2.0f) return set_error(PG_INVALID_ARG, "Gnufft: only gridos = 2 is supported");
  if (nx != ny) return set_error(PG_INVALID_ARG, "Gnufft: in-plane size must be square (nx == ny)");
  if (M >= (1ull << 32)) return set_error(PG_INVALID_ARG, "Gnufft: too many samples");
  for (uint64_t i = 0; i < M; ++i) {
    const float a = kx[i], b = ky[i], c = kz ? kz[i] : 0.f;
    if (!(std::isfinite(a) && std::isfinite(b) && std::isfinite(c)))
      return set_error(PG_INVALID_ARG, "Gnufft: non-finite k-space coordinate at %llu", (unsigned long long)i);
    // Gnufft.cpp:68-76 warns beyond 1.05*N/2; past that the 2-D adjoint
    // loop bounds of the reference are undefined, so reject instead.
    if (std::abs(a) > (nx / 2.0f) * 1.05f || std::abs(b) > (ny / 2.0f) * 1.05f ||
        (nz > 1 && std::abs(c) > (nz / 2.0f) * 1.05f))
      return set_error(PG_INVALID_ARG, "Gnufft: k-space trajectory out of range [-N/2, N/2] at %llu",
                       (unsigned long long)i);
  }
  auto p = std::make_unique<NufftPlan>();
  NufftGeom& g = p->g;
  g.dim = (nz == 1) ? 2 : 3;
  g.Nx = nx; g.Ny = ny; g.Nz = nz;
  g.Gx = (int)std::ceil(gridos * (float)nx);
  g.Gy = (int)std::ceil(gridos * (float)ny);
  if (g.Gx % 2) g.Gx += 1;
  if (g.Gy % 2) g.Gy += 1;
  g.Gz = (nz == 1) ? 1 : (int)std::ceil(gridos * (float)nz);
  if (g.Gx > 65535 || g.Gy > 65535 || g.Gz > 65535) return set_error(PG_INVALID_ARG, "Gnufft: grid too large");
  g.os = gridos;
  g.kw = 4.0f;
  std::vector<float> lut;
  kb_table(gridos, &lut, &g.beta);
  g.nlut = (int)lut.size();
  const int N3[3] = {nx, ny, nz};
  const int G3[3] = {g.Gx, g.Gy, g.Gz};
  for (int a = 0; a < 3; ++a) {
    const bool used = (a < 2) || g.dim == 3;
    g.pad_off[a] = used ? (int)(((float)N3[a] * gridos / 2.0f) - ((float)N3[a] / 2.0f)) : 0;
    g.crop_off[a] = used ? (int)(((float)G3[a] / 2.0f) - ((float)N3[a] / 2.0f)) : 0;
    g.fs[a] = used ? (int)std::floor(G3[a] / 2.0) : 0;
    g.ifs[a] = used ? ((a < 2) ? (int)std::ceil(G3[a] / 2.0) : (int)std::floor(G3[a] / 2.0)) : 0;
  }
  std::vector<float> deap(nx + ny + nz, 1.0f);
  for (int i = 0; i < nx; ++i) deap[i] = deapod_factor(i, nx, g.kw, g.beta, g.dim == 3);
  for (int i = 0; i < ny; ++i) deap[nx + i] = deapod_factor(i, ny, g.kw, g.beta, g.dim == 3);
  if (g.dim == 3)
    for (int i = 0; i < nz; ++i) deap[nx + ny + i] = deapod_factor(i, nz, g.kw, g.beta, true);
  p->M = M;
  PG_TRY(p->kx.upload(kx, M, s));
  PG_TRY(p->ky.upload(ky, M, s));
  std::vector<float> zeros;
  if (!kz) zeros.assign(M, 0.f);
  PG_TRY(p->kz.upload(kz ? kz : zeros.data(), M, s));
  PG_TRY(p->lut.upload(lut.data(), lut.size(), s));
  PG_TRY(p->deap.upload(deap.data(), deap.size(), s));
  PG_CUDA(cudaStreamSynchronize(s));
  // the unsegmented binning is built on first use (time-segmented operators never need it)
  *out = std::move(p);
  return PG_OK;
}

pg_status nufft_plain_binning(NufftPlan* p, cudaStream_t s) {
  if (p->plain) return PG_OK;
  return nufft_build_binning(p, 1, 1, nullptr, nullptr, &p->plain, s);
}

pg_status nufft_build_binning(NufftPlan* p, int L, int K, const int* l0_host, const float2* aa_host,
                              std::unique_ptr<Binning>* out, cudaStream_t s) {
  const NufftGeom& g = p->g;
  const uint64_t M = p->M;
  auto b = std::make_unique<Binning>();
  b->L = L; b->K = K; b->M = M;
  b->tile = choose_tiles(g);
  const TileShape& t = b->tile;
  const uint64_t ntiles = (uint64_t)t.ntx * t.nty * t.ntz;
  b->nkeys = ntiles * (uint64_t)L;
  if (b->nkeys >= (1ull << 32)) return set_error(PG_INVALID_ARG, "binning: too many bins");

  DevBuf<uint2> st_o;
  DevBuf<float> wxy_o, wz_o;
  DevBuf<uint32_t> key;
  DevBuf<int> l0d;
  PG_TRY(st_o.alloc(M));
  PG_TRY(wxy_o.alloc(M * 16));
  if (g.dim == 3) PG_TRY(wz_o.alloc(M * 8));
  PG_TRY(key.alloc(M));
  if (l0_host) PG_TRY(l0d.upload(l0_host, M, s));
  PG_LAUNCH(k_prepare, ceil_div(M, 256), 256, 0, s, g, M, p->kx.p, p->ky.p, p->kz.p, p->lut.p, t,
            l0_host ? l0d.p : nullptr, st_o.p, wxy_o.p, g.dim == 3 ? wz_o.p : nullptr, key.p);
  b->h_keys.resize(M);
  PG_CUDA(cudaMemcpyAsync(b->h_keys.data(), key.p, M * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));

  // Stable counting sort by key on the host (plan time, O(M + bins)).
  std::vector<uint64_t> cnt(b->nkeys + 1, 0);
  for (uint64_t i = 0; i < M; ++i) cnt[b->h_keys[i] + 1]++;
  for (uint64_t k = 0; k < b->nkeys; ++k) cnt[k + 1] += cnt[k];
  std::vector<uint64_t> pos(cnt.begin(), cnt.end() - 1);
  b->h_perm.resize(M);
  for (uint64_t i = 0; i < M; ++i) b->h_perm[pos[b->h_keys[i]]++] = (uint32_t)i;

  // Subproblems: each (segment window, tile) bin split into chunks.
  const int kMaxPerSub = (g.dim == 2) ? 512 : 256;
  std::vector<int4> subs;
  for (uint64_t k = 0; k < b->nkeys; ++k) {
    const uint64_t a = cnt[k], e = cnt[k + 1];
    if (a == e) continue;
    const int l = (int)(k / ntiles);
    const int tile = (int)(k % ntiles);
    for (uint64_t f = a; f < e; f += kMaxPerSub)
      subs.push_back(make_int4(tile, l, (int)f, (int)std::min<uint64_t>(kMaxPerSub, e - f)));
  }
  b->nsub = (int)subs.size();

  PG_TRY(b->perm.upload(b->h_perm.data(), M, s));
  PG_TRY(b->subprob.upload(subs.data(), subs.size(), s));
  PG_TRY(b->start.alloc(M));
  PG_TRY(b->wxy.alloc(M * 16));
  if (g.dim == 3) PG_TRY(b->wz.alloc(M * 8));
  PG_LAUNCH(k_permute, ceil_div(M, 256), 256, 0, s, M, g.dim, K, b->perm.p, st_o.p, wxy_o.p,
            g.dim == 3 ? wz_o.p : nullptr, b->start.p, b->wxy.p, g.dim == 3 ? b->wz.p : nullptr);
  if (l0_host) {
    std::vector<int> l0s(M);
    std::vector<float2> aas(M * (uint64_t)K);
    for (uint64_t j = 0; j < M; ++j) {
      const uint32_t i = b->h_perm[j];
      l0s[j] = l0_host[i];
      for (int q = 0; q < K; ++q) aas[j * K + q] = aa_host[(uint64_t)i * K + q];
    }
    PG_TRY(b->l0.upload(l0s.data(), M, s));
    PG_TRY(b->aa.upload(aas.data(), aas.size(), s));
  }
  PG_CUDA(cudaStreamSynchronize(s));
  *out = std::move(b);
  return PG_OK;
}

// ---------------------------------------------------------------------------
// Execution
// ---------------------------------------------------------------------------
static pg_status ensure_workspace(NufftPlan* p, int B, cufftHandle* h, cudaStream_t s) {
  const uint64_t G = p->g.ngrid();
  if (p->grids.n < (uint64_t)B * G) {
    PG_CUDA(cudaStreamSynchronize(s));  // queued work may still use the old workspace
    PG_TRY(p->grids.alloc((uint64_t)B * G));
  }
  auto it = p->ffts.find(B);
  if (it == p->ffts.end()) {
    cufftHandle hh;
    PG_CUFFT(cufftCreate(&hh));
    int n[3];
    int rank;
    if (p->g.dim == 2) { rank = 2; n[0] = p->g.Gx; n[1] = p->g.Gy; }
    else { rank = 3; n[0] = p->g.Gz; n[1] = p->g.Gx; n[2] = p->g.Gy; }
    size_t work = 0;
    PG_CUFFT(cufftSetAutoAllocation(hh, 0));
    cufftResult r = cufftMakePlanMany(hh, rank, n, nullptr, 1, (int)G, nullptr, 1, (int)G, CUFFT_C2C, B, &work);
    if (r != CUFFT_SUCCESS) {
      cufftDestroy(hh);
      return set_error(r == CUFFT_ALLOC_FAILED ? PG_OUT_OF_MEMORY : PG_CUFFT_ERROR, "cufftMakePlanMany: %d", (int)r);
    }
    if (work > p->fft_work.n) {
      // the old area may still be in use by queued transforms of this plan
      PG_CUDA(cudaStreamSynchronize(s));
      PG_TRY(p->fft_work.alloc(work));
    }
    it = p->ffts.emplace(B, hh).first;
  }
  PG_CUFFT(cufftSetWorkArea(it->second, p->fft_work.p));
  PG_CUFFT(cufftSetStream(it->second, s));
  *h = it->second;
  return PG_OK;
}

static int batch_coils(const NufftPlan* p, int C, int L) {
  const uint64_t per = (uint64_t)L * p->g.ngrid() * sizeof(float2);
  uint64_t cb = per ? p->budget_bytes / per : (uint64_t)C;
  if (cb < 1) cb = 1;
  return (int)std::min<uint64_t>(cb, (uint64_t)C);
}

pg_status nufft_forward(NufftPlan* p, const NufftBatch& b, const float2* x, float2* y, cudaStream_t s) {
  const NufftGeom& g = p->g;
  if (!b.bin) PG_TRY(nufft_plain_binning(p, s));
  const Binning* bin = b.bin ? b.bin : p->plain.get();
  const int L = bin->L, K = bin->K;
  const int Cb = batch_coils(p, b.C, L);
  const float scale = (g.dim == 2) ? (1.0f / (g.os * g.os)) : (float)(1.0 / (double)(g.os * g.os * g.os));
  const uint64_t G = g.ngrid();
  for (int c0 = 0; c0 < b.C; c0 += Cb) {
    const int nb = std::min(Cb, b.C - c0);
    const int B = nb * L;
    cufftHandle h;
    PG_TRY(ensure_workspace(p, B, &h, s));
    dim3 grid(ceil_div(G, 256), B);
    {
      ProfScope ps("pre", s);
      PG_LAUNCH(k_pre, grid, 256, 0, s, g, L, x, b.S, c0, b.E, b.Wo, p->deap.p, scale, p->grids.p);
    }
    {
      ProfScope ps("fft_fwd", s);
      PG_CUFFT(cufftExecC2C(h, reinterpret_cast<cufftComplex*>(p->grids.p),
                            reinterpret_cast<cufftComplex*>(p->grids.p), CUFFT_FORWARD));
    }
    float2* yc = y + (uint64_t)c0 * b.data_stride;
    const float2* aa = (L > 1 || bin->aa.p) ? bin->aa.p : nullptr;
    const int* l0 = bin->l0.p;
    ProfScope ps("gather", s);
    if (g.dim == 2)
      PG_LAUNCH(k_gather<2>, ceil_div(p->M, 128), 128, 0, s, g, p->M, bin->start.p, bin->wxy.p, bin->wz.p,
                bin->perm.p, l0, aa, K, L, p->grids.p, nb, yc, b.data_stride);
    else
      PG_LAUNCH(k_gather<3>, ceil_div(p->M, 128), 128, 0, s, g, p->M, bin->start.p, bin->wxy.p, bin->wz.p,
                bin->perm.p, l0, aa, K, L, p->grids.p, nb, yc, b.data_stride);
  }
  return PG_OK;
}

pg_status nufft_adjoint(NufftPlan* p, const NufftBatch& b, const float2* y, float2* x, cudaStream_t s) {
  const NufftGeom& g = p->g;
  if (!b.bin) PG_TRY(nufft_plain_binning(p, s));
  const Binning* bin = b.bin ? b.bin : p->plain.get();
  const int L = bin->L, K = bin->K;
  const int Cb = batch_coils(p, b.C, L);
  const float scale = (g.dim == 2) ? (1.0f / (g.os * g.os)) : (float)(1.0 / (double)(g.os * g.os * g.os));
  const uint64_t G = g.ngrid();
  const TileShape& t = bin->tile;
  const size_t plane_bytes = (size_t)t.PX * t.PY * t.PZ * 2 * sizeof(float);
  static int smem_optin = -1;
  if (smem_optin < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  }
  int Cc = (int)std::min<size_t>(4, (size_t)smem_optin / (plane_bytes * K));
  if (Cc < 1) return set_error(PG_INVALID_ARG, "adjoint: segment window K=%d too wide for shared memory", K);
  for (int c0 = 0; c0 < b.C; c0 += Cb) {
    const int nb = std::min(Cb, b.C - c0);
    const int B = nb * L;
    cufftHandle h;
    PG_TRY(ensure_workspace(p, B, &h, s));
    {
      ProfScope ps("zero", s);
      PG_CUDA(cudaMemsetAsync(p->grids.p, 0, (size_t)B * G * sizeof(float2), s));
    }
    const int cc = std::min(Cc, nb);
    const size_t smem = plane_bytes * K * cc;
    dim3 grid(bin->nsub, ceil_div(nb, cc));
    const float2* yc = y + (uint64_t)c0 * b.data_stride;
    const float2* aa = (L > 1 || bin->aa.p) ? bin->aa.p : nullptr;
    if (bin->nsub > 0) {
      ProfScope ps("spread", s);
      if (g.dim == 2) {
        PG_CUDA(cudaFuncSetAttribute(k_spread<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        PG_LAUNCH(k_spread<2>, grid, 256, smem, s, g, t, bin->subprob.p, bin->start.p, bin->wxy.p, bin->wz.p,
                  bin->perm.p, aa, K, L, yc, b.data_stride, nb, cc, p->grids.p);
      } else {
        PG_CUDA(cudaFuncSetAttribute(k_spread<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        PG_LAUNCH(k_spread<3>, grid, 256, smem, s, g, t, bin->subprob.p, bin->start.p, bin->wxy.p, bin->wz.p,
                  bin->perm.p, aa, K, L, yc, b.data_stride, nb, cc, p->grids.p);
      }
    }
    {
      ProfScope ps("fft_adj", s);
      PG_CUFFT(cufftExecC2C(h, reinterpret_cast<cufftComplex*>(p->grids.p),
                            reinterpret_cast<cufftComplex*>(p->grids.p), CUFFT_INVERSE));
    }
    const int acc = (b.accumulate || c0 > 0) ? 1 : 0;
    ProfScope ps("post", s);
    PG_LAUNCH(k_post, ceil_div(g.nimg(), 256), 256, 0, s, g, nb, L, p->grids.p, b.S, c0, b.E, b.WoH, p->deap.p,
              scale, acc, x);
  }
  return PG_OK;
}

}  // namespace pg
