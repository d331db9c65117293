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
#include <mutex>
#include <tuple>

#include "pg_binsort.cuh"
#include "pg_fftpass.cuh"
#include "pg_kb.cuh"
#include "pg_nufft.cuh"
#include "pg_profile.cuh"

namespace pg {

PG_DEFINE_CHECK_WORD()


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
  int lo, hi;
  const float s = kb_window(k, n_img, os, kw, &lo, &hi);
  const int st = (hi - lo == 8) ? lo + 1 : lo;
  const float kw2 = __fmul_rn(kw, kw);
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const int c = st + a;
    w[a] = (c >= lo && c <= hi) ? kb_weight(s, c, os, kw2, lut, nlut) : 0.0f;
  }
  return st;
}

__device__ __forceinline__ int wrap(int v, int n) {
  v %= n;
  return v < 0 ? v + n : v;
}

// Per-sample preparation (original order): tap starts, weights and bin key.
// The stored weights carry the +-1 checkerboard that replaces the shifts:
// for even G, ifftshift(FFT(fftshift(u))) = c (-1)^k FFT((-1)^n u) with
// c = prod_d (-1)^(G_d/2), so the gather and spread work on the unshifted
// (centred) grid, where the reference's clamped windows never wrap.
__global__ void k_prepare(NufftGeom g, uint64_t M, const float* __restrict__ kx, const float* __restrict__ ky,
                          const float* __restrict__ kz, const float* __restrict__ lut, TileShape t,
                          const int* __restrict__ l0, uint2* __restrict__ start, float* __restrict__ wxy,
                          float* __restrict__ wz, uint32_t* __restrict__ key) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  float w[8];
  const float c = g.sign_c;
  const int sx = axis_taps(kx[i], g.Nx, g.os, g.kw, lut, g.nlut, w);
#pragma unroll
  for (int a = 0; a < 8; ++a) wxy[i * 16 + a] = ((sx + a) & 1) ? -c * w[a] : c * w[a];
  const int sy = axis_taps(ky[i], g.Ny, g.os, g.kw, lut, g.nlut, w);
#pragma unroll
  for (int a = 0; a < 8; ++a) wxy[i * 16 + 8 + a] = ((sy + a) & 1) ? -w[a] : w[a];
  int sz = 0;
  if (g.dim == 3) {
    sz = axis_taps(kz[i], g.Nz, g.os, g.kw, lut, g.nlut, w);
#pragma unroll
    for (int a = 0; a < 8; ++a) wz[i * 8 + a] = ((sz + a) & 1) ? -w[a] : w[a];
  }
  start[i] = make_uint2((uint32_t)sx | ((uint32_t)sy << 16), (uint32_t)sz);
  const int tx = sx / t.TX, ty = sy / t.TY, tz = sz / t.TZ;
  const int l = l0 ? l0[i] : 0;
  key[i] = (uint32_t)((((uint64_t)l * t.ntz + tz) * t.ntx + tx) * t.nty + ty);
}

__global__ void k_permute(uint64_t M, int dim, int K, const uint32_t* __restrict__ perm,
                          const uint2* __restrict__ start_in, const float* __restrict__ wxy_in,
                          const float* __restrict__ wz_in, uint2* __restrict__ start_out,
                          float* __restrict__ wxy_out, float* __restrict__ wz_out, const int* __restrict__ l0_in,
                          const float2* __restrict__ aa_in, int* __restrict__ l0_out, float2* __restrict__ aa_out) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  const uint32_t i = perm[j];
  if (l0_in) {
    l0_out[j] = l0_in[i];
    for (int q = 0; q < K; ++q) aa_out[j * K + q] = aa_in[(uint64_t)i * K + q];
  }
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

__device__ __forceinline__ int parity3(int a, int b, int c) { return (a + b + c) & 1; }

// ---------------------------------------------------------------------------
// Forward pre-kernel: deapodize, coil map, shot phase and segment phase,
// times the (-1)^(x+y+z) checkerboard, into the image region of the centred
// forward-input grid.  The zero-pad border of that buffer is cleared once
// when it is allocated and never written, so only N^d cells per grid move.
// One thread per (pixel, grid of the batch).
// ---------------------------------------------------------------------------
__global__ void k_pre(NufftGeom g, int L, const float2* __restrict__ x, const float2* __restrict__ S, int c0,
                      const float2* __restrict__ E, const float2* __restrict__ Wo, const float* __restrict__ deapf,
                      float2* __restrict__ grids) {
  pdl_wait();
  const uint64_t N = g.nimg();
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int b = blockIdx.y;           // grid within the batch
  const int c = b / L, l = b - c * L;
  const int iy = (int)(p % g.Ny);
  const int ix = (int)((p / g.Ny) % g.Nx);
  const int iz = (int)(p / ((uint64_t)g.Ny * g.Nx));
  const int my = iy + g.pad_off[1];
  const int mx = ix + g.pad_off[0];
  const int mz = (g.dim == 3) ? iz + g.pad_off[2] : 0;
  const uint64_t q = (uint64_t)my + (uint64_t)g.Gy * ((uint64_t)mx + (uint64_t)g.Gx * mz);
  float2 v = x[p];
  if (S) {
    const float2 sv = S[(uint64_t)(c0 + c) * N + p];
    v = E ? cmul(v, cmul(sv, E[p])) : cmul(sv, v);
  }
  if (Wo) v = cmul(Wo[(uint64_t)l * N + p], v);
  const float f = parity3(mx, my, mz) ? -deapf[p] : deapf[p];
  v = make_float2(v.x * f, v.y * f);
  grids[(uint64_t)b * g.ngrid() + q] = v;
}

// Adjoint preparation in one launch: zero the batch's grids (n4 float4
// words) and write, in binned sample order, the value each sample spreads
// into each segment of its window, vs[c][s][j] = conj(AA(s, l0+j)) y_c[perm s].
__global__ void k_adjoint_prep(uint64_t n4, float4* __restrict__ grids, int nb, uint64_t M, int K,
                               const uint32_t* __restrict__ perm, const float2* __restrict__ aa,
                               const float2* __restrict__ y, uint64_t dstride, float2* __restrict__ vs) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (uint64_t i = t0; i < n4; i += stride) grids[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int c = 0; c < nb; ++c)
    for (uint64_t s = t0; s < M; s += stride) {
      const float2 d = y[(uint64_t)c * dstride + perm[s]];
      float2* o = vs + ((uint64_t)c * M + s) * K;
      if (aa)
        for (int j = 0; j < K; ++j) o[j] = cmul(cconj(aa[s * K + j]), d);
      else
        o[0] = d;
    }
}

// Asynchronous global -> shared copies (cp.async; 16 bytes bypass L1).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Padded extent along y (the fastest axis) such that 4 x-rows of 8 y-taps
// land in 32 distinct banks: PY = 8 or 24 (mod 32).
__host__ __device__ constexpr int padded_y(int T) {
  int py = T + 8;
  while ((py % 32) != 8 && (py % 32) != 24) ++py;
  return py;
}

// Compile-time tile geometry: every shared-memory address in the gridding
// loops is a per-sample base plus an immediate offset.
template <int DIM, int T>
struct TileGeo {
  static constexpr int TZ = (DIM == 3) ? T : 1;
  static constexpr int PX = T + 8;
  static constexpr int PY = padded_y(T);
  static constexpr int PZ = (DIM == 3) ? T + 8 : 1;
  static constexpr int PLANE = PX * PY;
  static constexpr int CELLS = PLANE * PZ;
};

// Device work queue of the persistent spread launch: items are (subproblem,
// coil chunk) pairs, subproblems largest first.  Each block takes the next
// item until none is left; the block that finds the queue empty last resets
// it for the next launch.  Returns the item, or -1.
__device__ __forceinline__ int next_item(unsigned* q, int nitems) {
  __shared__ int item;
  __syncthreads();   // the previous item's shared memory is no longer in use
  if (threadIdx.x == 0) {
    int it = (int)atomicAdd(&q[0], 1u);
    if (it >= nitems) {
      it = -1;
      if (atomicAdd(&q[1], 1u) == gridDim.x - 1) { q[0] = 0u; q[1] = 0u; }
    }
    item = it;
  }
  __syncthreads();
  return item;
}

// ---------------------------------------------------------------------------
// Forward interpolation, tiled: one block per (subproblem, coil chunk), in 2-D
// two for subproblems of more than kGatherHalf samples.  The
// padded tiles of the subproblem's KP segment grids for CC coils are staged in
// shared memory as complex cells ([c][j][PZ][PX][PY]).  Then one thread per
// sample reads its 8^d cells of every (coil, segment) plane and sums them in
// the reference's order (x outer, y inner, gridding.cpp:275-289) with paired
// fma; no cross-lane reduction is needed, and consecutive samples of a warp
// often share their window (spiral readouts are oversampled along the arm),
// so their shared-memory reads broadcast.  The segment interpolator AA is
// applied per coil on the way out.
// ---------------------------------------------------------------------------
constexpr int kGatherHalf = 128;   // 2-D subproblems above this are gathered by two blocks

template <int DIM, int T, int CC, int KP>
__global__ void __launch_bounds__(128) k_gather(NufftGeom g, TileShape t, const int4* __restrict__ sub,
                                                const uint2* __restrict__ start, const float* __restrict__ wxy,
                                                const float* __restrict__ wz, const uint32_t* __restrict__ perm,
                                                const float2* __restrict__ aa, int K, int L,
                                                const float2* __restrict__ grids, int Cb,
                                                float2* __restrict__ data, uint64_t dstride) {
  pdl_wait();
  using TG = TileGeo<DIM, T>;
  constexpr int CELLS = TG::CELLS, PY = TG::PY, PX = TG::PX, PLANE = TG::PLANE;
  extern __shared__ __align__(16) float2 sm2[];   // [c*KP + j][PZ][PX][PY] complex cells
  // In 2-D two blocks share a subproblem of more than kGatherHalf samples,
  // one per half (more blocks to cover the staging latency; each stages the
  // tile); the second block of a smaller subproblem has nothing to do.
  constexpr int SPLIT = (DIM == 2) ? 2 : 1;
  const int4 sp = sub[blockIdx.x / SPLIT];
  const int part = blockIdx.x % SPLIT;
  const int head = (SPLIT == 2 && sp.w > kGatherHalf) ? (sp.w + 1) / 2 : sp.w;
  const int first = sp.z + part * head, count = part ? sp.w - head : head;
  if (count <= 0) return;
  const int cfirst = blockIdx.y * CC;
  const int ncl = min(CC, Cb - cfirst);
  const int tile = sp.x, lseg = sp.y;
  const int ty = tile % t.nty;
  const int txz = tile / t.nty;
  const int tx = txz % t.ntx;
  const int tz = txz / t.ntx;
  const int x0 = tx * T, y0 = ty * T, z0 = tz * TG::TZ;
  const uint64_t G = g.ngrid();
  // cell pairs (y, y+1) with asynchronous 16-byte copies: PY, y0 and Gy are
  // even, so a pair is in the grid or outside it as a whole and both of its
  // addresses are 16-byte aligned
  static_assert(PY % 2 == 0 && CELLS % 2 == 0, "cell pairs");
  for (int t2 = threadIdx.x; t2 < CELLS / 2; t2 += blockDim.x) {
    const int q = 2 * t2;
    const int pyy = q % PY;
    const int pxx = (q / PY) % PX;
    const int pzz = q / PLANE;
    const int gy = y0 + pyy, gx = x0 + pxx, gz = z0 + pzz;
    const bool in = gy < g.Gy && gx < g.Gx && gz < g.Gz;
    const uint64_t idx = (uint64_t)gy + (uint64_t)g.Gy * ((uint64_t)gx + (uint64_t)g.Gx * gz);
#pragma unroll
    for (int c = 0; c < CC; ++c)
#pragma unroll
      for (int j = 0; j < KP; ++j) {
        float2* d = &sm2[(c * KP + j) * CELLS + q];
        if (in && c < ncl && j < K)
          cp_async16(d, &grids[((uint64_t)(cfirst + c) * L + lseg + j) * G + idx]);
        else
          *reinterpret_cast<float4*>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
  }
  cp_async_wait_all();
  __syncthreads();
  const int end = first + count;
  for (int s = first + threadIdx.x; s < end; s += blockDim.x) {
    const uint2 st = start[s];
    const int ox = (int)(st.x & 0xffff) - x0, oy = (int)(st.x >> 16) - y0;
    if (!PG_CHECK(ox >= 0 && ox < T && oy >= 0 && oy < T &&
                      (DIM == 2 || ((int)st.y - z0 >= 0 && (int)st.y - z0 < TG::TZ)),
                  PG_SITE_GATHER_WINDOW, ox * 65536 + oy))
      continue;
    const float4* w4 = reinterpret_cast<const float4*>(wxy + (uint64_t)s * 16);
    const float4 wa = w4[0], wb = w4[1], wc = w4[2], wd = w4[3];
    const float wxr[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    const float wyr[8] = {wc.x, wc.y, wc.z, wc.w, wd.x, wd.y, wd.z, wd.w};
    float2 acc[CC * KP];
#pragma unroll
    for (int i = 0; i < CC * KP; ++i) acc[i] = make_float2(0.f, 0.f);
    const float2* base = sm2 + ox * PY + oy;
    if (DIM == 2) {
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int d = 0; d < 8; ++d) {
          const float w = wxr[r] * wyr[d];
          const float2 w2 = make_float2(w, w);
#pragma unroll
          for (int cj = 0; cj < CC * KP; ++cj) acc[cj] = __ffma2_rn(w2, base[cj * CELLS + r * PY + d], acc[cj]);
        }
    } else {
      const int oz = (int)st.y - z0;
      const float* wzz = wz + (uint64_t)s * 8;
      const float2* bz = base + oz * PLANE;
#pragma unroll 1
      for (int e = 0; e < 8; ++e, bz += PLANE) {
        const float wze = wzz[e];
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
          for (int d = 0; d < 8; ++d) {
            const float w = wxr[r] * wyr[d] * wze;
            const float2 w2 = make_float2(w, w);
#pragma unroll
            for (int cj = 0; cj < CC * KP; ++cj) acc[cj] = __ffma2_rn(w2, bz[cj * CELLS + r * PY + d], acc[cj]);
          }
      }
    }
    const uint32_t o = perm[s];
    if (!PG_CHECK(o < dstride, PG_SITE_GATHER_PERM, o)) continue;
#pragma unroll
    for (int c = 0; c < CC; ++c) {
      if (c >= ncl) break;
      float2 out = acc[c * KP];
      if (aa) {
        out = cmul(acc[c * KP], aa[(uint64_t)s * K]);
#pragma unroll
        for (int j = 1; j < KP; ++j)
          if (j < K) out = cadd(out, cmul(acc[c * KP + j], aa[(uint64_t)s * K + j]));
      }
      data[(uint64_t)(cfirst + c) * dstride + o] = out;
    }
  }
}

// ---------------------------------------------------------------------------
// Adjoint spread, persistent: as many blocks as fit on the device take
// (subproblem, coil chunk) items from a device work queue, largest first.
//  1. The subproblem's samples are staged in shared memory with coalesced
//     loads: tap starts, tap weights and, per (coil, segment) plane, the value
//     v = conj(AA) * y the sample spreads.
//  2. Each plane gets a power-of-two scale 2^e from the largest |re| or |im|
//     of its values, chosen so that every single contribution w * v * 2^e is
//     below 2^22 in magnitude and the sum of all of them in one cell (at most
//     one per sample, at most 256 << extra samples) stays below 2^30.
//  3. A warp spreads one sample at a time into the padded tile, lane =
//     (y-tap, x-tap pair), with 32-bit integer shared atomics (native, unlike
//     float shared atomics).  The integer of a contribution is formed by one
//     fma against the constant 1.5 * 2^23: for |x| < 2^22 the sum lands in
//     [2^23, 2^24), where the float grid spacing is 1, so the fma rounds w*v
//     to the nearest integer, held in the low mantissa bits.  Integer sums do
//     not depend on the order of the atomics, so the result is deterministic.
//  4. Each nonzero tile cell is flushed to the centred grid with one vector
//     atomic, scaled back by 2^-e.
// Tile layout [coil][segment][re|im][PZ][PX][PY], PY = 8 (mod 32): a warp's
// 32 lanes (8 y-taps x 4 x-taps) hit 32 distinct banks.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int fixed_point(float w, float v) {
  constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23, float bits 0x4B400000
  return __float_as_int(__fmaf_rn(w, v, kMagic)) - 0x4B400000;
}

// Staged weights per sample in the spread: wx[8], wy[8] and, in 3-D, wz[8].
__host__ __device__ constexpr int spread_wrow(int dim) { return dim == 2 ? 16 : 24; }

template <int DIM, int T, int NP>
__global__ void __launch_bounds__(256) k_spread(NufftGeom g, TileShape t, const int4* __restrict__ sub,
                                                const uint2* __restrict__ start, const float* __restrict__ wxy,
                                                const float* __restrict__ wz, const float2* __restrict__ vs,
                                                uint64_t M, int K, int L, int c0, int cc, int smax, float wmax,
                                                float2* __restrict__ grids, unsigned* __restrict__ queue,
                                                int nchunks, int nitems) {
  pdl_wait();
  using TG = TileGeo<DIM, T>;
  constexpr int CELLS = TG::CELLS, PY = TG::PY, PX = TG::PX, PLANE = TG::PLANE;
  constexpr int WROW = spread_wrow(DIM);   // staged weights per sample: wx[8] wy[8] (wz[8])
  extern __shared__ __align__(16) int smi[];
  __shared__ unsigned vmax[16];
  __shared__ float scale[16], inv_scale[16];
  // planes per block: NP when fixed at compile time, else cc x K
  const int np = (NP > 0) ? NP : cc * K;
  // The tile planes are zeroed once here; afterwards each item's flush zeroes
  // every cell as it reads it (one thread per cell), and the scale step
  // resets the plane maxima it has read (next_item's barrier orders both).
  {
    int4* z = reinterpret_cast<int4*>(smi);
    for (int q = threadIdx.x; q < (np * 2 * CELLS) / 4; q += blockDim.x) z[q] = make_int4(0, 0, 0, 0);
  }
  if (threadIdx.x < 16) vmax[threadIdx.x] = 0u;
  for (int item; (item = next_item(queue, nitems)) >= 0;) {
  const int4 sp = sub[item / nchunks];
  const int cfirst = c0 + (item % nchunks) * cc;
  const int tile = sp.x, first = sp.z, count = sp.w;
  const int lseg = sp.y;
  if (!PG_CHECK(count <= smax, PG_SITE_SPREAD_COUNT, count)) continue;   // uniform across the block
  const int ty = tile % t.nty;
  const int txz = tile / t.nty;
  const int tx = txz % t.ntx;
  const int tz = txz / t.ntx;
  const int x0 = tx * T, y0 = ty * T, z0 = tz * TG::TZ;
  const int tid = threadIdx.x;
  float* sw = reinterpret_cast<float*>(smi + (size_t)np * 2 * CELLS);
  float2* sv = reinterpret_cast<float2*>(sw + (size_t)smax * WROW);
  uint2* sst = reinterpret_cast<uint2*>(sv + (size_t)smax * np);

  // 1. staging: asynchronous copies straight into shared memory (no register
  // round trip; every copy of the item is in flight before the one wait)
  constexpr int R4 = WROW / 4;
  for (int q = tid; q < count * R4; q += blockDim.x) {
    const int i = q / R4, a = q % R4;
    const float4* src = (a < 4) ? reinterpret_cast<const float4*>(wxy + (uint64_t)(first + i) * 16) + a
                                : reinterpret_cast<const float4*>(wz + (uint64_t)(first + i) * 8) + (a - 4);
    cp_async16(reinterpret_cast<float4*>(sw + i * WROW) + a, src);
  }
  for (int i = tid; i < count; i += blockDim.x) cp_async8(&sst[i], &start[first + i]);
  // sv[i][c*K + j] = vs[cfirst + c][first + i][j]: for each coil of the block
  // the block's samples are one contiguous run of count*K values
  const int nk = count * K;
  for (int c = 0; c < cc; ++c) {
    const float2* src = vs + ((uint64_t)(cfirst + c) * M + first) * K;
    for (int r = tid; r < nk; r += blockDim.x) {
      const int i = (K == 1) ? r : (K == 2) ? (r >> 1) : r / K;
      cp_async8(&sv[i * np + c * K + (r - i * K)], &src[r]);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  // largest |re| or |im| per plane (non-negative floats order like their bit
  // patterns): a register maximum per thread, then one atomic per warp
  for (int pl = 0; pl < np; ++pl) {
    unsigned m = 0u;
    for (int i = tid; i < count; i += blockDim.x) {
      const float2 v = sv[i * np + pl];
      m = max(m, __float_as_uint(fmaxf(fabsf(v.x), fabsf(v.y))));
    }
    m = __reduce_max_sync(0xffffffffu, m);
    if ((tid & 31) == 0 && m) atomicMax(&vmax[pl], m);
  }
  __syncthreads();

  // 2. per-plane scale
  if (tid < 16) {
    int extra = 0;
    while (count > (256 << extra)) ++extra;
    const float B = __uint_as_float(vmax[tid]) * wmax * 1.0001f;
    int e = 0;
    if (B > 0.f) {
      frexpf(B, &e);                       // B < 2^e
      e = 22 - e - extra;                  // B * 2^e' < 2^(22 - extra)
    }
    scale[tid] = ldexpf(1.f, e);
    inv_scale[tid] = ldexpf(1.f, -e);
    vmax[tid] = 0u;                        // for the next item
  }
  __syncthreads();
  // the scale is applied to each value as the spread reads it (exact: a power of two)

  // 3. spread
  const int warp = tid >> 5, lane = tid & 31;
  constexpr int NW = 8;
  const int dy = lane & 7, dx = lane >> 3;
  if (DIM == 2 && NP > 0) {
    // Each warp walks a contiguous run of samples.  Samples are in readout
    // order within a bin, so consecutive ones often share their window start;
    // a lane then keeps hitting the same two cells, so it sums the run's
    // contributions in registers (paired fp32 fma, fixed order) and issues
    // the shared atomics once per run of equal starts, rounding the run sum
    // to the integer grid.  Integer sums of the runs do not depend on the
    // order of the atomics, so the result is deterministic.
    constexpr int NPC = NP > 0 ? NP : 1;
    float scp[NPC];
#pragma unroll
    for (int pl = 0; pl < NPC; ++pl) scp[pl] = scale[pl];
    const int per = (count + NW - 1) / NW;
    const int i0 = warp * per, i1 = min(count, i0 + per);
    float2 a0[NPC], a1[NPC];              // (re, im) at tap dx and dx + 4
    uint32_t prev = 0xffffffffu;
    int* b = smi;
    bool open = false;
    auto flush_run = [&]() {
#pragma unroll
      for (int pl = 0; pl < NPC; ++pl) {
        atomicAdd(b + (2 * pl) * CELLS, __float2int_rn(a0[pl].x));
        atomicAdd(b + (2 * pl + 1) * CELLS, __float2int_rn(a0[pl].y));
        atomicAdd(b + (2 * pl) * CELLS + 4 * PY, __float2int_rn(a1[pl].x));
        atomicAdd(b + (2 * pl + 1) * CELLS + 4 * PY, __float2int_rn(a1[pl].y));
      }
    };
    for (int i = i0; i < i1; ++i) {
      const uint2 st = sst[i];
      if (st.x != prev) {                  // uniform across the warp
        if (open) flush_run();
        open = false;
        prev = st.x;
        const int ox = (int)(st.x & 0xffff) - x0, oy = (int)(st.x >> 16) - y0;
        if (!PG_CHECK(ox >= 0 && ox < T && oy >= 0 && oy < T, PG_SITE_SPREAD_WINDOW, ox * 65536 + oy)) {
          prev = 0xffffffffu;
          continue;
        }
        open = true;
        b = smi + (ox + dx) * PY + oy + dy;
#pragma unroll
        for (int pl = 0; pl < NPC; ++pl) a0[pl] = a1[pl] = make_float2(0.f, 0.f);
      }
      const float* w = sw + i * WROW;
      const float wyv = w[8 + dy];
      const float w0 = w[dx] * wyv, w1 = w[dx + 4] * wyv;
      const float2 w0v = make_float2(w0, w0), w1v = make_float2(w1, w1);
      const float2* vi = sv + i * NPC;
#pragma unroll
      for (int pl = 0; pl < NPC; ++pl) {
        const float2 u = vi[pl];
        const float2 v = make_float2(u.x * scp[pl], u.y * scp[pl]);
        a0[pl] = __ffma2_rn(w0v, v, a0[pl]);
        a1[pl] = __ffma2_rn(w1v, v, a1[pl]);
      }
    }
    if (open) flush_run();
  } else {
    for (int i = warp; i < count; i += NW) {
      const uint2 st = sst[i];
      const int ox = (int)(st.x & 0xffff) - x0, oy = (int)(st.x >> 16) - y0;
      if (!PG_CHECK(ox >= 0 && ox < T && oy >= 0 && oy < T &&
                        (DIM == 2 || ((int)st.y - z0 >= 0 && (int)st.y - z0 < TG::TZ)),
                    PG_SITE_SPREAD_WINDOW, ox * 65536 + oy))
        continue;                          // uniform across the warp
      const float* w = sw + i * WROW;
      const float wyv = w[8 + dy];
      const float w0 = w[dx] * wyv, w1 = w[dx + 4] * wyv;
      int* b = smi + (ox + dx) * PY + oy + dy;
      const float2* vi = sv + i * np;
      if (DIM == 2) {
#pragma unroll
        for (int pl = 0; pl < np; ++pl) {
          const float2 u = vi[pl];
          const float sc = scale[pl];
          const float2 v = make_float2(u.x * sc, u.y * sc);
          atomicAdd(b + (2 * pl) * CELLS, fixed_point(w0, v.x));
          atomicAdd(b + (2 * pl + 1) * CELLS, fixed_point(w0, v.y));
          atomicAdd(b + (2 * pl) * CELLS + 4 * PY, fixed_point(w1, v.x));
          atomicAdd(b + (2 * pl + 1) * CELLS + 4 * PY, fixed_point(w1, v.y));
        }
      } else {
        b += ((int)st.y - z0) * PLANE;
#pragma unroll 1
        for (int e = 0; e < 8; ++e, b += PLANE) {
          const float wzv = w[16 + e];
          if (wzv == 0.f) continue;          // uniform across the warp
          const float w0e = w0 * wzv, w1e = w1 * wzv;
#pragma unroll
          for (int pl = 0; pl < np; ++pl) {
            const float2 u = vi[pl];
            const float sc = scale[pl];
            const float2 v = make_float2(u.x * sc, u.y * sc);
            atomicAdd(b + (2 * pl) * CELLS, fixed_point(w0e, v.x));
            atomicAdd(b + (2 * pl + 1) * CELLS, fixed_point(w0e, v.y));
            atomicAdd(b + (2 * pl) * CELLS + 4 * PY, fixed_point(w1e, v.x));
            atomicAdd(b + (2 * pl + 1) * CELLS + 4 * PY, fixed_point(w1e, v.y));
          }
        }
      }
    }
  }
  __syncthreads();

  // 4. flush
  const uint64_t G = g.ngrid();
  for (int q = tid; q < CELLS; q += blockDim.x) {
    const int pyy = q % PY;
    const int pxx = (q / PY) % PX;
    const int pzz = q / PLANE;
    const int gy = y0 + pyy, gx = x0 + pxx, gz = z0 + pzz;
    const bool inside = gy < g.Gy && gx < g.Gx && gz < g.Gz;
    const uint64_t idx = (uint64_t)gy + (uint64_t)g.Gy * ((uint64_t)gx + (uint64_t)g.Gx * gz);
    int pl = 0;
    for (int c = 0; c < cc; ++c)
      for (int j = 0; j < K; ++j, ++pl) {
        int* pr = smi + (pl * 2) * CELLS;
        const int re = pr[q], im = pr[CELLS + q];
        if (re != 0 || im != 0) {
          pr[q] = 0;                       // zero for the next item
          pr[CELLS + q] = 0;
          if (inside)
            atomicAdd(grids + ((uint64_t)(cfirst + c) * L + lseg + j) * G + idx,
                      make_float2((float)re * inv_scale[pl], (float)im * inv_scale[pl]));
        }
      }
  }
  }
}

// ---------------------------------------------------------------------------
// 2-D adjoint spread with the adjoint preparation folded in, for segment
// windows of KK <= 2 (Hanning time segmentation, or none).  Persistent like
// k_spread: blocks take (subproblem, coil chunk of CC) items from the device
// work queue, largest first.  Per item:
//  1. staging: tap weights and window starts by cp.async; the values
//     v = conj(AA(s, l0 + j)) * y_c[perm s] read straight from the data
//     vector (no intermediate array), with their largest |re| or |im|
//     reduced in registers, then per warp;
//  2. the bounding box of the item's windows, and one power-of-two scale
//     2^e for all of the item's planes, chosen as in k_spread so that every
//     single contribution w * v * 2^e is below 2^22 and every cell sum below
//     2^30; it multiplies the y weight of each sample (exact);
//  3. the spread: each warp walks a contiguous run of samples, lane = (y tap,
//     x-tap pair); runs of equal window start are summed in registers with
//     paired fp32 fma (two planes per 16-byte value load) and rounded once to
//     the integer grid, one int32 shared atomic per tap, plane and run;
//  4. the flush: the bounding box only, two cells per 16-byte vector atomic;
//     each cell is zeroed as it is read, so the tile is zero for the next item.
// The grids are cleared before the launch (a memset).  Integer tile sums do
// not depend on the order of the atomics; the flush into the grid is a float
// vector atomic per cell pair.
// Shared memory: tile planes [NP][re|im][PX][PY] int32, weights [smax][16]
// f32, values [smax][NP2] float4 (two planes each), window starts [smax] u32.
// ---------------------------------------------------------------------------
// Blocks per SM the folded spread's register budget is sized for: its shared
// memory admits 5 items of up to 4 planes (44 KB each at 256 samples) and 3 of
// 8 planes.
__host__ __device__ constexpr int spread2d_min_blocks(int np) { return np <= 4 ? 5 : 3; }

template <int T, int CC, int KK>
__global__ void __launch_bounds__(256, spread2d_min_blocks(CC * KK))
    k_spread2d(NufftGeom g, TileShape t, const int4* __restrict__ sub,
                                                  const uint2* __restrict__ start, const float* __restrict__ wxy,
                                                  const uint32_t* __restrict__ perm, const float2* __restrict__ aa,
                                                  const float2* __restrict__ y, uint64_t dstride, int nb, int L,
                                                  int smax, float wmax, float2* __restrict__ grids,
                                                  unsigned* __restrict__ queue, int nchunks, int nitems) {
  pdl_wait();
  using TG = TileGeo<2, T>;
  constexpr int CELLS = TG::CELLS, PY = TG::PY;
  constexpr int NP = CC * KK;          // planes per item
  constexpr int NP2 = (NP + 1) / 2;    // 16-byte value slots per sample
  static_assert(CC == 1 || CC == 2 || CC == 4, "coils per item: 1, 2 or 4");
  static_assert(PY % 2 == 0 && CELLS % 2 == 0, "cell pairs");
  extern __shared__ __align__(16) int smi[];
  __shared__ unsigned vmax;
  __shared__ int box[4];               // window starts: min x, max x, min y, max y (tile coordinates)
  __shared__ int s_item;
  __shared__ float s_scale[2];         // 2^e and 2^-e of the current item
  const int tid = threadIdx.x;
  int* tile = smi;
  float* sw = reinterpret_cast<float*>(smi + NP * 2 * CELLS);
  float4* sv = reinterpret_cast<float4*>(sw + (size_t)smax * 16);
  float2* sv2 = reinterpret_cast<float2*>(sv);
  uint32_t* sst = reinterpret_cast<uint32_t*>(sv + (size_t)smax * NP2);
  for (int q = tid; q < NP * 2 * CELLS / 4; q += blockDim.x) reinterpret_cast<int4*>(tile)[q] = make_int4(0, 0, 0, 0);
  for (;;) {
    __syncthreads();                   // the previous item's shared memory is no longer in use
    if (tid == 0) {
      int it = (int)atomicAdd(&queue[0], 1u);
      if (it >= nitems) {
        it = -1;
        if (atomicAdd(&queue[1], 1u) == gridDim.x - 1) { queue[0] = 0u; queue[1] = 0u; }
      }
      s_item = it;
      vmax = 0u;
      box[0] = box[2] = 0x7fffffff;
      box[1] = box[3] = -1;
    }
    __syncthreads();
    const int item = s_item;
    if (item < 0) break;
    const int4 sp = sub[item / nchunks];
    const int cfirst = (item % nchunks) * CC;
    const int ncl = min(CC, nb - cfirst);
    const int tile_i = sp.x, lseg = sp.y, first = sp.z, count = sp.w;
    if (!PG_CHECK(count <= smax, PG_SITE_SPREAD_COUNT, count)) continue;   // uniform across the block
    const int x0 = (tile_i / t.nty) * T, y0 = (tile_i % t.nty) * T;

    // 1. staging
    for (int q = tid; q < count * 4; q += blockDim.x) {
      const int i = q >> 2, a = q & 3;
      cp_async16(reinterpret_cast<float4*>(sw + i * 16) + a,
                 reinterpret_cast<const float4*>(wxy + (uint64_t)(first + i) * 16) + a);
    }
    for (int i = tid; i < count; i += blockDim.x) cp_async4(&sst[i], &start[first + i].x);
    {
      const int c = tid % CC;
      float m = 0.f;
      for (int i = tid / CC; i < count; i += blockDim.x / CC) {
        const uint64_t s = (uint64_t)(first + i);
        float2 d = make_float2(0.f, 0.f);
        if (c < ncl) {
          const uint32_t ps = perm[s];
          if (PG_CHECK(ps < dstride, PG_SITE_SPREAD2D_PERM, ps)) d = y[(uint64_t)(cfirst + c) * dstride + ps];
        }
#pragma unroll
        for (int j = 0; j < KK; ++j) {
          const float2 v = aa ? cmul(cconj(aa[s * KK + j]), d) : d;
          m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
          sv2[(size_t)i * 2 * NP2 + c * KK + j] = v;
        }
      }
      const unsigned u = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
      if ((tid & 31) == 0 && u) atomicMax(&vmax, u);
    }
    cp_async_wait_all();
    __syncthreads();

    // 2. bounding box of the windows and the item's scale
    {
      int xlo = 0x7fffffff, xhi = -1, ylo = 0x7fffffff, yhi = -1;
      for (int i = tid; i < count; i += blockDim.x) {
        const uint32_t st = sst[i];
        const int ox = (int)(st & 0xffff) - x0, oy = (int)(st >> 16) - y0;
        xlo = min(xlo, ox); xhi = max(xhi, ox);
        ylo = min(ylo, oy); yhi = max(yhi, oy);
      }
      xlo = __reduce_min_sync(0xffffffffu, xlo);
      xhi = __reduce_max_sync(0xffffffffu, xhi);
      ylo = __reduce_min_sync(0xffffffffu, ylo);
      yhi = __reduce_max_sync(0xffffffffu, yhi);
      if ((tid & 31) == 0 && xhi >= 0) {
        atomicMin(&box[0], xlo); atomicMax(&box[1], xhi);
        atomicMin(&box[2], ylo); atomicMax(&box[3], yhi);
      }
    }
    if (tid == 0) {
      int extra = 0;
      while (count > (256 << extra)) ++extra;
      const float B = __uint_as_float(vmax) * wmax * 1.0001f;
      int e = 0;
      if (B > 0.f) {
        frexpf(B, &e);                 // B < 2^e
        e = 22 - e - extra;            // B * 2^e' < 2^(22 - extra)
      }
      s_scale[0] = ldexpf(1.f, e);
      s_scale[1] = ldexpf(1.f, -e);
    }
    __syncthreads();
    const float sc = s_scale[0], inv = s_scale[1];

    // 3. spread
    {
      const int warp = tid >> 5, lane = tid & 31;
      constexpr int NW = 8;
      const int dy = lane & 7, dx = lane >> 3;
      const int per = (count + NW - 1) / NW;
      const int i0 = warp * per, i1 = min(count, i0 + per);
      float2 a0[NP], a1[NP];           // (re, im) at tap dx and dx + 4
      uint32_t prev = 0xffffffffu;
      int* b = tile;
      bool open = false;
      auto flush_run = [&]() {
#pragma unroll
        for (int pl = 0; pl < NP; ++pl) {
          if (pl / KK >= ncl) break;
          atomicAdd(b + (2 * pl) * CELLS, __float2int_rn(a0[pl].x));
          atomicAdd(b + (2 * pl + 1) * CELLS, __float2int_rn(a0[pl].y));
          atomicAdd(b + (2 * pl) * CELLS + 4 * PY, __float2int_rn(a1[pl].x));
          atomicAdd(b + (2 * pl + 1) * CELLS + 4 * PY, __float2int_rn(a1[pl].y));
        }
      };
      for (int i = i0; i < i1; ++i) {
        const uint32_t st = sst[i];
        if (st != prev) {              // uniform across the warp
          if (open) flush_run();
          open = false;
          prev = st;
          const int ox = (int)(st & 0xffff) - x0, oy = (int)(st >> 16) - y0;
          if (!PG_CHECK(ox >= 0 && ox < T && oy >= 0 && oy < T, PG_SITE_SPREAD2D_WINDOW, ox * 65536 + oy)) {
            prev = 0xffffffffu;
            continue;
          }
          open = true;
          b = tile + (ox + dx) * PY + oy + dy;
#pragma unroll
          for (int pl = 0; pl < NP; ++pl) a0[pl] = a1[pl] = make_float2(0.f, 0.f);
        }
        const float* w = sw + i * 16;
        const float wyv = w[8 + dy] * sc;
        const float w0 = w[dx] * wyv, w1 = w[dx + 4] * wyv;
        const float2 w0v = make_float2(w0, w0), w1v = make_float2(w1, w1);
        if constexpr (NP % 2 == 0) {
          const float4* vi = sv + (size_t)i * NP2;
#pragma unroll
          for (int q = 0; q < NP2; ++q) {
            const float4 u = vi[q];
            const float2 ua = make_float2(u.x, u.y), ub = make_float2(u.z, u.w);
            a0[2 * q] = __ffma2_rn(w0v, ua, a0[2 * q]);
            a1[2 * q] = __ffma2_rn(w1v, ua, a1[2 * q]);
            a0[2 * q + 1] = __ffma2_rn(w0v, ub, a0[2 * q + 1]);
            a1[2 * q + 1] = __ffma2_rn(w1v, ub, a1[2 * q + 1]);
          }
        } else {
          const float2* vi = sv2 + (size_t)i * 2 * NP2;
#pragma unroll
          for (int pl = 0; pl < NP; ++pl) {
            const float2 u = vi[pl];
            a0[pl] = __ffma2_rn(w0v, u, a0[pl]);
            a1[pl] = __ffma2_rn(w1v, u, a1[pl]);
          }
        }
      }
      if (open) flush_run();
    }
    __syncthreads();

    // 4. flush the bounding box, two cells (y, y + 1) per vector atomic
    {
      constexpr int PX = TG::PX, PYP = PY / 2;   // cell pairs per padded row
      const int bx0 = box[0], bx1 = box[1] + 7, by0 = box[2] >> 1, by1 = (box[3] + 7) >> 1;
      const uint64_t G = g.ngrid();
      for (int q = tid; q < PX * PYP; q += blockDim.x) {
        const int px = q / PYP, pp = q - px * PYP;
        if (px < bx0 || px > bx1 || pp < by0 || pp > by1) continue;
        const int py = 2 * pp;
        const int cell = px * PY + py;
        const int gx = x0 + px, gy = y0 + py;
        const bool inside = gx < g.Gx && gy < g.Gy;
        const uint64_t idx = (uint64_t)gy + (uint64_t)g.Gy * (uint64_t)gx;
#pragma unroll
        for (int pl = 0; pl < NP; ++pl) {
          const int c = pl / KK, j = pl % KK;
          if (c >= ncl) break;
          int2* pr = reinterpret_cast<int2*>(tile + (2 * pl) * CELLS + cell);
          int2* pi = reinterpret_cast<int2*>(tile + (2 * pl + 1) * CELLS + cell);
          const int2 re = *pr, im = *pi;
          if ((re.x | re.y | im.x | im.y) != 0) {
            *pr = make_int2(0, 0);
            *pi = make_int2(0, 0);
            if (inside)
              atomicAdd(reinterpret_cast<float4*>(grids + ((uint64_t)(cfirst + c) * L + lseg + j) * G + idx),
                        make_float4((float)re.x * inv, (float)im.x * inv, (float)re.y * inv, (float)im.y * inv));
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Adjoint post-kernel: crop the centred grid, undo the checkerboard,
// deapodize, apply WoH, combine segments and coils.  CP x LP lanes share one
// pixel: lane (c, h) takes coils c, c+CP, ... and segments h, h+LP, ...; the
// lanes' images are added with a fixed xor-butterfly (deterministic).
// ---------------------------------------------------------------------------
template <int CP, int LP>
__global__ void k_post(NufftGeom g, int Cb, int L, const float2* __restrict__ grids, const float2* __restrict__ S,
                       int c0, const float2* __restrict__ E, const float2* __restrict__ WoH,
                       const float* __restrict__ deapf, int accumulate, float2* __restrict__ x) {
  pdl_wait();
  constexpr int LN = CP * LP;
  const uint64_t N = g.nimg();
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int ln = (int)(t % LN);
  const int cl = ln / LP, hl = ln % LP;
  const uint64_t p = t / LN;
  float2 acc = make_float2(0.f, 0.f);
  if (p < N) {
    const int iy = (int)(p % g.Ny);
    const int ix = (int)((p / g.Ny) % g.Nx);
    const int iz = (int)(p / ((uint64_t)g.Ny * g.Nx));
    const int gy = iy + g.crop_off[1];
    const int gx = ix + g.crop_off[0];
    const int gz = (g.dim == 3) ? iz + g.crop_off[2] : 0;
    const uint64_t q = (uint64_t)gy + (uint64_t)g.Gy * ((uint64_t)gx + (uint64_t)g.Gx * gz);
    const uint64_t G = g.ngrid();
    const float f = parity3(gx, gy, gz) ? -deapf[p] : deapf[p];
    const float2 e = E ? cconj(E[p]) : make_float2(1.f, 0.f);
    for (int c = cl; c < Cb; c += CP) {
      float2 img = make_float2(0.f, 0.f);
#pragma unroll 4
      for (int l = hl; l < L; l += LP) {
        float2 v = grids[((uint64_t)c * L + l) * G + q];
        v = make_float2(v.x * f, v.y * f);
        if (WoH) v = cmul(v, WoH[(uint64_t)l * N + p]);
        img = cadd(img, v);
      }
      if (S) {
        const float2 sv = S[(uint64_t)(c0 + c) * N + p];
        img = E ? cmul(cmul(cconj(sv), e), img) : cmul(img, cconj(sv));
      }
      acc = cadd(acc, img);
    }
  }
#pragma unroll
  for (int o = LN / 2; o >= 1; o >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
  }
  if (p < N && ln == 0) x[p] = accumulate ? cadd(x[p], acc) : acc;
}

// ---------------------------------------------------------------------------
// Plan construction
// ---------------------------------------------------------------------------
namespace {
struct FftKey;
}
static void fft_release_plan(const NufftGeom& g, int B, cufftHandle h, size_t work);

NufftPlan::~NufftPlan() {
  for (auto& kv : ffts) fft_release_plan(g, kv.first, kv.second.first, kv.second.second);
}

NufftTune NufftTune::defaults() {
  NufftTune t;
  auto env = [](const char* n, int d) {
    const char* v = getenv(n);
    return (v && *v) ? atoi(v) : d;
  };
  t.tile2d = env("PG_TILE2D", t.tile2d);
  t.tile3d = env("PG_TILE3D", t.tile3d);
  t.submax2d = env("PG_SUBMAX2D", t.submax2d);
  t.submax3d = env("PG_SUBMAX3D", t.submax3d);
  t.spread_cc = env("PG_SPREAD_CC", t.spread_cc);
  t.gather_cc = env("PG_GATHER_CC", t.gather_cc);
  return t;
}

// Tile edges with compiled gridding kernels: 16 or 32 in 2-D, 8 in 3-D.
static bool tile_supported(int dim, int T) { return dim == 2 ? (T == 16 || T == 32) : T == 8; }

static TileShape choose_tiles(const NufftGeom& g, const NufftTune& tu) {
  TileShape t{};
  if (g.dim == 2) {
    t.TX = t.TY = tile_supported(2, tu.tile2d) ? tu.tile2d : 16; t.TZ = 1;
    t.PX = t.TX + 8; t.PY = padded_y(t.TY); t.PZ = 1;
  } else {
    t.TX = t.TY = t.TZ = tile_supported(3, tu.tile3d) ? tu.tile3d : 8;
    t.PX = t.TX + 8; t.PY = padded_y(t.TY); t.PZ = t.TZ + 8;
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
  p->tune = NufftTune::defaults();
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
  // The table depends only on the oversampling factor (fixed at 2 here):
  // build it once per process.
  static const std::pair<std::vector<float>, float> kTable = [] {
    std::pair<std::vector<float>, float> t;
    kb_table(2.0f, &t.first, &t.second);
    return t;
  }();
  const std::vector<float>& lut = kTable.first;
  g.beta = kTable.second;
  g.nlut = (int)lut.size();
  const int N3[3] = {nx, ny, nz};
  const int G3[3] = {g.Gx, g.Gy, g.Gz};
  g.sign_c = 1.0f;
  for (int a = 0; a < 3; ++a) {
    const bool used = (a < 2) || g.dim == 3;
    if (used && (G3[a] % 2)) return set_error(PG_INVALID_ARG, "Gnufft: oversampled grid must be even");
    if (used && ((G3[a] / 2) % 2)) g.sign_c = -g.sign_c;
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
  p->lut_max = *std::max_element(lut.begin(), lut.end());
  PG_TRY(p->deap.upload(deap.data(), deap.size(), s));
  // power-of-two 2N grids run the pruned, fused FFT passes; PG_CUFFT=1 keeps cuFFT
  {
    const char* e = getenv("PG_CUFFT");
    p->own_fft = fftpass_supported(g) && !(e && e[0] == '1');
    if (p->own_fft) PG_TRY(fftpass_twiddles(g, &p->tw2d, s));
  }
  // Per-voxel deapodization factor 1/(OS^d k), k the product of the axis
  // factors in float as the reference forms it; 0 where k is NaN (the
  // reference zeroes those voxels, griddingSupport.cpp:265-278).
  {
    const float scale = (g.dim == 2) ? (1.0f / (gridos * gridos)) : (float)(1.0 / (double)(gridos * gridos * gridos));
    std::vector<float> f((uint64_t)nx * ny * nz);
    for (int z = 0; z < nz; ++z)
      for (int xx = 0; xx < nx; ++xx)
        for (int yy = 0; yy < ny; ++yy) {
          float k = deap[xx] * deap[nx + yy];
          if (g.dim == 3) k = k * deap[nx + ny + z];
          f[(uint64_t)yy + (uint64_t)ny * ((uint64_t)xx + (uint64_t)nx * z)] =
              (k == k) ? (float)((double)scale / (double)k) : 0.f;
        }
    PG_TRY(p->deapf.upload(f.data(), f.size(), s));
  }
  PG_CUDA(cudaStreamSynchronize(s));
  // the unsegmented binning is built on first use (time-segmented operators never need it)
  *out = std::move(p);
  return PG_OK;
}

pg_status nufft_plan_share(const NufftPlan& src, std::unique_ptr<NufftPlan>* out) {
  auto p = std::make_unique<NufftPlan>();
  p->g = src.g;
  p->tune = src.tune;
  p->M = src.M;
  p->lut_max = src.lut_max;
  p->budget_bytes = src.budget_bytes;
  p->kx.borrow(src.kx);
  p->ky.borrow(src.ky);
  p->kz.borrow(src.kz);
  p->lut.borrow(src.lut);
  p->deap.borrow(src.deap);
  p->deapf.borrow(src.deapf);
  p->own_fft = src.own_fft;
  p->tw2d.borrow(src.tw2d);
  if (src.plain) p->plain = binning_share(*src.plain);
  *out = std::move(p);
  return PG_OK;
}

std::unique_ptr<Binning> binning_share(const Binning& b) {
  auto o = std::make_unique<Binning>();
  o->K = b.K; o->L = b.L; o->M = b.M; o->tile = b.tile;
  o->nsub = b.nsub; o->submax = b.submax; o->nkeys = b.nkeys;
  o->perm.borrow(b.perm);
  o->keys.borrow(b.keys);
  o->start.borrow(b.start);
  o->wxy.borrow(b.wxy);
  o->wz.borrow(b.wz);
  o->l0.borrow(b.l0);
  o->aa.borrow(b.aa);
  o->subprob.borrow(b.subprob);
  return o;
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
  b->tile = choose_tiles(g, p->tune);
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

  // Stable counting sort by key on the device (bit-exact against a CPU one).
  DevBuf<uint32_t> starts_d;
  PG_TRY(b->perm.alloc(M));
  PG_TRY(starts_d.alloc(b->nkeys));
  PG_TRY(bin_sort(key.p, M, b->nkeys, b->perm.p, starts_d.p, s));
  std::vector<uint32_t> starts(b->nkeys);
  PG_CUDA(cudaMemcpyAsync(starts.data(), starts_d.p, b->nkeys * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));

  // Subproblems: each (segment window, tile) bin split into chunks.
  const int kMaxPerSub = (g.dim == 2) ? p->tune.submax2d : p->tune.submax3d;
  std::vector<int4> subs;
  for (uint64_t k = 0; k < b->nkeys; ++k) {
    const uint64_t a = starts[k], e = (k + 1 < b->nkeys) ? starts[k + 1] : M;
    if (a == e) continue;
    const int l = (int)(k / ntiles);
    const int tile = (int)(k % ntiles);
    for (uint64_t f = a; f < e; f += kMaxPerSub)
      subs.push_back(make_int4(tile, l, (int)f, (int)std::min<uint64_t>(kMaxPerSub, e - f)));
  }
  // Largest subproblems first: blocks are dispatched roughly in index order,
  // so the small ones fill the last wave instead of trailing it.
  std::stable_sort(subs.begin(), subs.end(), [](const int4& a, const int4& c) { return a.w > c.w; });
  b->nsub = (int)subs.size();
  b->submax = kMaxPerSub;

  PG_TRY(b->subprob.upload(subs.data(), subs.size(), s));
  PG_TRY(b->start.alloc(M));
  PG_TRY(b->wxy.alloc(M * 16));
  if (g.dim == 3) PG_TRY(b->wz.alloc(M * 8));
  DevBuf<float2> aa_d;
  if (l0_host) {
    PG_TRY(aa_d.upload(aa_host, M * (uint64_t)K, s));
    PG_TRY(b->l0.alloc(M));
    PG_TRY(b->aa.alloc(M * (uint64_t)K));
  }
  PG_LAUNCH(k_permute, ceil_div(M, 256), 256, 0, s, M, g.dim, K, b->perm.p, st_o.p, wxy_o.p,
            g.dim == 3 ? wz_o.p : nullptr, b->start.p, b->wxy.p, g.dim == 3 ? b->wz.p : nullptr,
            l0_host ? l0d.p : nullptr, l0_host ? aa_d.p : nullptr, l0_host ? b->l0.p : nullptr,
            l0_host ? b->aa.p : nullptr);
  b->keys = std::move(key);
  PG_CUDA(cudaStreamSynchronize(s));
  *out = std::move(b);
  return PG_OK;
}

// ---------------------------------------------------------------------------
// Execution
// ---------------------------------------------------------------------------
// Process-wide pool of cuFFT plans keyed by (grid shape, batch).  Plans are
// created without an internal work area; a NufftPlan checks handles out on
// first use, supplies its own work area and stream on every execution, and
// returns them when destroyed, so serving many requests of recurring shapes
// does not re-plan.
namespace {
struct FftKey {
  int rank, n0, n1, n2, batch;
  bool operator<(const FftKey& o) const {
    return std::tie(rank, n0, n1, n2, batch) < std::tie(o.rank, o.n0, o.n1, o.n2, o.batch);
  }
};
std::mutex g_fft_mu;
std::map<FftKey, std::vector<std::pair<cufftHandle, size_t>>> g_fft_free;

FftKey fft_key(const NufftGeom& g, int B) {
  return g.dim == 2 ? FftKey{2, g.Gx, g.Gy, 0, B} : FftKey{3, g.Gz, g.Gx, g.Gy, B};
}

pg_status fft_acquire(const FftKey& k, cufftHandle* h, size_t* work) {
  {
    std::lock_guard<std::mutex> lk(g_fft_mu);
    auto it = g_fft_free.find(k);
    if (it != g_fft_free.end() && !it->second.empty()) {
      *h = it->second.back().first;
      *work = it->second.back().second;
      it->second.pop_back();
      return PG_OK;
    }
  }
  cufftHandle hh;
  PG_CUFFT(cufftCreate(&hh));
  int n[3] = {k.n0, k.n1, k.n2};
  const int G = k.n0 * k.n1 * (k.rank == 3 ? k.n2 : 1);
  size_t w = 0;
  cufftResult r = cufftSetAutoAllocation(hh, 0);
  if (r == CUFFT_SUCCESS) r = cufftMakePlanMany(hh, k.rank, n, nullptr, 1, G, nullptr, 1, G, CUFFT_C2C, k.batch, &w);
  if (r != CUFFT_SUCCESS) {
    cufftDestroy(hh);
    return set_error(r == CUFFT_ALLOC_FAILED ? PG_OUT_OF_MEMORY : PG_CUFFT_ERROR, "cufftMakePlanMany: %d", (int)r);
  }
  *h = hh;
  *work = w;
  return PG_OK;
}

void fft_release(const FftKey& k, cufftHandle h, size_t work) {
  std::lock_guard<std::mutex> lk(g_fft_mu);
  g_fft_free[k].emplace_back(h, work);
}
}  // namespace

static void fft_release_plan(const NufftGeom& g, int B, cufftHandle h, size_t work) {
  fft_release(fft_key(g, B), h, work);
}

// Grid workspace for B grids and, unless the plan runs its own FFT passes
// (h == nullptr), the pooled cuFFT plan for a batch of B.
static pg_status ensure_workspace(NufftPlan* p, int B, cufftHandle* h, cudaStream_t s) {
  const uint64_t G = p->g.ngrid();
  if (p->work->grids.n < (uint64_t)B * G) {
    PG_CUDA(cudaStreamSynchronize(s));  // queued work may still use the old workspace
    PG_TRY(p->work->grids.alloc((uint64_t)B * G));
  }
  if (!h) return PG_OK;
  auto it = p->ffts.find(B);
  if (it == p->ffts.end()) {
    cufftHandle hh;
    size_t work = 0;
    PG_TRY(fft_acquire(fft_key(p->g, B), &hh, &work));
    if (work > p->work->fft_work.n) {
      // the old area may still be in use by queued transforms of this plan
      PG_CUDA(cudaStreamSynchronize(s));
      pg_status st = p->work->fft_work.alloc(work);
      if (st != PG_OK) { fft_release(fft_key(p->g, B), hh, work); return st; }
    }
    it = p->ffts.emplace(B, std::make_pair(hh, work)).first;
  }
  PG_CUFFT(cufftSetWorkArea(it->second.first, p->work->fft_work.p));
  PG_CUFFT(cufftSetStream(it->second.first, s));
  *h = it->second.first;
  return PG_OK;
}

// The adjoint's spread target on the 2-D own-FFT path: B zeroed grids.
static pg_status ensure_adjoint_grids(NufftPlan* p, int B, cudaStream_t s) {
  const uint64_t n = (uint64_t)B * p->g.ngrid();
  NufftWork& w = *p->work;
  if (w.agrids.n < n || !w.agrids.p) {
    if (w.agrids.p) PG_CUDA(cudaStreamSynchronize(s));
    PG_TRY(w.agrids.alloc(n));
    w.agrids_clean = false;
  }
  if (!w.agrids_clean) {
    PG_CUDA(cudaMemsetAsync(w.agrids.p, 0, w.agrids.n * sizeof(float2), s));
    w.agrids_clean = true;
  }
  return PG_OK;
}

// Forward input grids: the image region is rewritten by every forward, the
// zero-pad border only here, when the buffer is (re)allocated.  cuFFT's
// out-of-place C2C transform leaves its input unchanged.
static pg_status ensure_forward_input(NufftPlan* p, int B, cudaStream_t s) {
  const uint64_t n = (uint64_t)B * p->g.ngrid();
  if (p->work->fin.n >= n && p->work->fin.p) return PG_OK;
  if (p->work->fin.p) PG_CUDA(cudaStreamSynchronize(s));
  PG_TRY(p->work->fin.alloc(n));
  PG_CUDA(cudaMemsetAsync(p->work->fin.p, 0, n * sizeof(float2), s));
  return PG_OK;
}

// The 2-D adjoint spreads into a grid set that its first inverse FFT pass
// zeroes after reading (a full pass over contiguous rows, where the stores
// are nearly free).  The 3-D first pass reads z columns across slabs, where
// the same stores cost more than a separate clearing, so 3-D keeps clearing
// the forward's grids in the adjoint preparation.
static bool self_clearing(const NufftPlan& p) { return p.own_fft && p.g.dim == 2; }

static int batch_coils(const NufftPlan* p, int C, int L) {
  // 2-D own FFT passes: forward grids and the adjoint's self-clearing spread target
  const uint64_t per = (uint64_t)L * p->g.ngrid() * sizeof(float2) * (self_clearing(*p) ? 2 : 1);
  uint64_t cb = per ? p->budget_bytes / per : (uint64_t)C;
  if (cb < 1) cb = 1;
  return (int)std::min<uint64_t>(cb, (uint64_t)C);
}

static int smem_optin_bytes() {
  static const int v = [] {
    int dev = 0, a = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&a, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return a;
  }();
  return v;
}

// The spread kernels' shared memory depends on the bin size, which differs
// between plans; worker threads of the request server launch them
// concurrently.  Raising the allowed dynamic shared memory per launch would
// let one thread lower it between another thread's raise and launch, so it is
// set once per kernel to the device's opt-in limit (less its static shared
// memory), which covers every launch.
static pg_status allow_full_dynamic_smem(const void* kernel) {
  static std::mutex mu;
  static std::map<const void*, bool> done;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(kernel)) return PG_OK;
  cudaFuncAttributes fa{};
  PG_CUDA(cudaFuncGetAttributes(&fa, kernel));
  const int dyn = smem_optin_bytes() - (int)fa.sharedSizeBytes;
  PG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
  done[kernel] = true;
  return PG_OK;
}

// Blocks of a persistent launch: as many as fit on the device at
// once (cached per kernel and shared-memory size), at most one per item.
static int persistent_blocks(const void* kernel, size_t smem, int nitems) {
  static std::mutex mu;
  static std::map<std::pair<const void*, size_t>, int> cache;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find({kernel, smem});
    if (it != cache.end()) {
      per_sm = it->second;
    } else {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem) != cudaSuccess) {
        cudaGetLastError();
        per_sm = 1;
      }
      cache[{kernel, smem}] = per_sm = std::max(1, per_sm);
    }
  }
  return std::max(1, std::min(nitems, per_sm * sm_count()));
}

// The work-queue words of the plan's persistent spread launches (zero between launches).
static pg_status ensure_queue(NufftPlan* p, cudaStream_t s) {
  if (p->work->queue.p) return PG_OK;
  PG_TRY(p->work->queue.alloc(2));
  PG_CUDA(cudaMemsetAsync(p->work->queue.p, 0, 2 * sizeof(unsigned), s));
  return PG_OK;
}

// Tiled gather launch: choose the padded segment count KP and the coils per
// block CC so that the staged tiles fit in shared memory and the per-thread
// accumulators (2*CC*KP floats) stay at most 32.
template <int DIM, int T, int CC, int KP>
static pg_status gather_launch_one(NufftPlan* p, const Binning* bin, const float2* aa, int nb, float2* y,
                                   uint64_t dstride, cudaStream_t s) {
  const size_t smem = (size_t)CC * KP * 2 * TileGeo<DIM, T>::CELLS * sizeof(float);
  PG_CUDA(cudaFuncSetAttribute(k_gather<DIM, T, CC, KP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // a static grid: the persistent work-queue form measured ~4 % slower here
  dim3 grid(bin->nsub * (DIM == 2 ? 2 : 1), ceil_div(nb, CC));
  PG_LAUNCH_PDL((k_gather<DIM, T, CC, KP>), grid, 128, smem, s, p->g, bin->tile, bin->subprob.p, bin->start.p,
            bin->wxy.p, bin->wz.p, bin->perm.p, aa, bin->K, bin->L, p->work->grids.p, nb, y, dstride);
  return PG_OK;
}

template <int DIM, int T>
static pg_status launch_gather_t(NufftPlan* p, const Binning* bin, const float2* aa, int nb, float2* y,
                                 uint64_t dstride, cudaStream_t s) {
  const int K = bin->K;
  const int KP = K <= 1 ? 1 : K <= 2 ? 2 : K <= 4 ? 4 : 8;
  const size_t pair = (size_t)TileGeo<DIM, T>::CELLS * 2 * sizeof(float);
  const size_t limit = (size_t)smem_optin_bytes() - 6144;  // static reduction buffer + margin
  int CC = std::max(1, std::min(4, p->tune.gather_cc));
  while (CC > 1 && (CC >= 2 * nb || 2 * CC * KP > 32 || (size_t)CC * KP * pair > limit)) CC >>= 1;
  if ((size_t)CC * KP * pair > limit || 2 * CC * KP > 32)
    return set_error(PG_INVALID_ARG, "forward: segment window K=%d too wide for shared memory", K);
  switch (KP * 10 + CC) {
    case 11: return gather_launch_one<DIM, T, 1, 1>(p, bin, aa, nb, y, dstride, s);
    case 12: return gather_launch_one<DIM, T, 2, 1>(p, bin, aa, nb, y, dstride, s);
    case 14: return gather_launch_one<DIM, T, 4, 1>(p, bin, aa, nb, y, dstride, s);
    case 21: return gather_launch_one<DIM, T, 1, 2>(p, bin, aa, nb, y, dstride, s);
    case 22: return gather_launch_one<DIM, T, 2, 2>(p, bin, aa, nb, y, dstride, s);
    case 24: return gather_launch_one<DIM, T, 4, 2>(p, bin, aa, nb, y, dstride, s);
    case 41: return gather_launch_one<DIM, T, 1, 4>(p, bin, aa, nb, y, dstride, s);
    case 42: return gather_launch_one<DIM, T, 2, 4>(p, bin, aa, nb, y, dstride, s);
    case 44: return gather_launch_one<DIM, T, 4, 4>(p, bin, aa, nb, y, dstride, s);
    case 81: return gather_launch_one<DIM, T, 1, 8>(p, bin, aa, nb, y, dstride, s);
    case 82: return gather_launch_one<DIM, T, 2, 8>(p, bin, aa, nb, y, dstride, s);
  }
  return set_error(PG_INVALID_ARG, "forward: unsupported tiling (K=%d)", K);
}

static pg_status launch_gather(NufftPlan* p, const Binning* bin, const float2* aa, int nb, float2* y,
                               uint64_t dstride, cudaStream_t s) {
  if (p->g.dim == 3) return launch_gather_t<3, 8>(p, bin, aa, nb, y, dstride, s);
  if (bin->tile.TX == 32) return launch_gather_t<2, 32>(p, bin, aa, nb, y, dstride, s);
  return launch_gather_t<2, 16>(p, bin, aa, nb, y, dstride, s);
}

// Spread launch arguments shared by every instantiation.
struct SpreadArgs {
  const float2* vs;
  int c0, cc, nchunks;
  float wmax;
  size_t smem;
};

template <int DIM, int T, int NP>
static pg_status spread_launch_np(NufftPlan* p, const Binning* bin, const SpreadArgs& a, float2* target,
                                  cudaStream_t s) {
  PG_TRY(allow_full_dynamic_smem((const void*)k_spread<DIM, T, NP>));
  const int nitems = bin->nsub * a.nchunks;
  PG_TRY(ensure_queue(p, s));
  const int blocks = persistent_blocks((const void*)k_spread<DIM, T, NP>, a.smem, nitems);
  PG_LAUNCH_PDL((k_spread<DIM, T, NP>), blocks, 256, a.smem, s, p->g, bin->tile, bin->subprob.p, bin->start.p,
            bin->wxy.p, bin->wz.p, a.vs, bin->M, bin->K, bin->L, a.c0, a.cc, bin->submax, a.wmax, target,
            p->work->queue.p, a.nchunks, nitems);
  return PG_OK;
}

// Planes per block (coils x segments) with an unrolled kernel; others use the
// runtime-loop instantiation (NP = 0).
template <int DIM, int T>
static pg_status spread_launch_t(NufftPlan* p, const Binning* bin, const SpreadArgs& a, float2* target,
                                 cudaStream_t s) {
  switch (a.cc * bin->K) {
    case 1: return spread_launch_np<DIM, T, 1>(p, bin, a, target, s);
    case 2: return spread_launch_np<DIM, T, 2>(p, bin, a, target, s);
    case 3: return spread_launch_np<DIM, T, 3>(p, bin, a, target, s);
    case 4: return spread_launch_np<DIM, T, 4>(p, bin, a, target, s);
    case 6: return spread_launch_np<DIM, T, 6>(p, bin, a, target, s);
    case 8: return spread_launch_np<DIM, T, 8>(p, bin, a, target, s);
  }
  return spread_launch_np<DIM, T, 0>(p, bin, a, target, s);
}

static pg_status launch_spread(NufftPlan* p, const Binning* bin, const SpreadArgs& a, float2* target,
                               cudaStream_t s) {
  if (p->g.dim == 3) return spread_launch_t<3, 8>(p, bin, a, target, s);
  if (bin->tile.TX == 32) return spread_launch_t<2, 32>(p, bin, a, target, s);
  return spread_launch_t<2, 16>(p, bin, a, target, s);
}

// Shared memory of k_spread2d: tile planes, staged weights, values and starts.
static size_t spread2d_smem(int T, int np, int smax) {
  const int px = T + 8, py = padded_y(T);
  return (size_t)np * 2 * px * py * sizeof(int) +
         (size_t)smax * (16 * sizeof(float) + (size_t)((np + 1) / 2) * sizeof(float4) + sizeof(uint32_t));
}

template <int T, int CC, int KK>
static pg_status spread2d_launch(NufftPlan* p, const Binning* bin, const float2* aa, const float2* y,
                                 uint64_t dstride, int nb, float wmax, float2* target, cudaStream_t s) {
  const size_t smem = spread2d_smem(T, CC * KK, bin->submax);
  PG_TRY(allow_full_dynamic_smem((const void*)k_spread2d<T, CC, KK>));
  const int nchunks = (nb + CC - 1) / CC;
  const int nitems = bin->nsub * nchunks;
  PG_TRY(ensure_queue(p, s));
  const int blocks = persistent_blocks((const void*)k_spread2d<T, CC, KK>, smem, nitems);
  PG_LAUNCH_PDL((k_spread2d<T, CC, KK>), blocks, 256, smem, s, p->g, bin->tile, bin->subprob.p, bin->start.p, bin->wxy.p,
            bin->perm.p, aa, y, dstride, nb, bin->L, bin->submax, wmax, target, p->work->queue.p, nchunks, nitems);
  return PG_OK;
}

template <int T>
static pg_status spread2d_launch_t(NufftPlan* p, const Binning* bin, int cc, const float2* aa, const float2* y,
                                   uint64_t dstride, int nb, float wmax, float2* target, cudaStream_t s) {
  switch (cc * 10 + bin->K) {
    case 11: return spread2d_launch<T, 1, 1>(p, bin, aa, y, dstride, nb, wmax, target, s);
    case 21: return spread2d_launch<T, 2, 1>(p, bin, aa, y, dstride, nb, wmax, target, s);
    case 41: return spread2d_launch<T, 4, 1>(p, bin, aa, y, dstride, nb, wmax, target, s);
    case 12: return spread2d_launch<T, 1, 2>(p, bin, aa, y, dstride, nb, wmax, target, s);
    case 22: return spread2d_launch<T, 2, 2>(p, bin, aa, y, dstride, nb, wmax, target, s);
    case 42: return spread2d_launch<T, 4, 2>(p, bin, aa, y, dstride, nb, wmax, target, s);
  }
  return set_error(PG_INVALID_ARG, "adjoint: no folded spread for %d coils x K=%d", cc, bin->K);
}

// Post-kernel launch: CP coil lanes x LP segment lanes per pixel (powers of
// two, at most 8 lanes).
template <int CP, int LP>
static pg_status post_launch(NufftPlan* p, int nb, int L, const NufftBatch& b, const float2* WoH,
                             const float2* grids, int c0, int acc, float2* x, cudaStream_t s) {
  const uint64_t N = p->g.nimg();
  PG_LAUNCH_PDL((k_post<CP, LP>), ceil_div(N * CP * LP, 256), 256, 0, s, p->g, nb, L, grids, b.S, c0, b.E, WoH,
            p->deapf.p, acc, x);
  return PG_OK;
}

// nb coils starting at coil c0 of the batch's maps, whose grids start at
// `grids`; x (+)= their image.
static pg_status launch_post(NufftPlan* p, int nb, int L, const NufftBatch& b, const float2* WoH,
                             const float2* grids, int c0, int acc, float2* x, cudaStream_t s) {
  const int cp = nb >= 8 ? 8 : nb >= 4 ? 4 : nb >= 2 ? 2 : 1;
  const int lp = std::min(8 / cp, L >= 4 ? 4 : L >= 2 ? 2 : 1);
  switch (cp * 10 + lp) {
    case 81: return post_launch<8, 1>(p, nb, L, b, WoH, grids, c0, acc, x, s);
    case 42: return post_launch<4, 2>(p, nb, L, b, WoH, grids, c0, acc, x, s);
    case 41: return post_launch<4, 1>(p, nb, L, b, WoH, grids, c0, acc, x, s);
    case 24: return post_launch<2, 4>(p, nb, L, b, WoH, grids, c0, acc, x, s);
    case 22: return post_launch<2, 2>(p, nb, L, b, WoH, grids, c0, acc, x, s);
    case 21: return post_launch<2, 1>(p, nb, L, b, WoH, grids, c0, acc, x, s);
    case 14: return post_launch<1, 4>(p, nb, L, b, WoH, grids, c0, acc, x, s);
    case 12: return post_launch<1, 2>(p, nb, L, b, WoH, grids, c0, acc, x, s);
    default: return post_launch<1, 1>(p, nb, L, b, WoH, grids, c0, acc, x, s);
  }
}

pg_status nufft_forward(NufftPlan* p, const NufftBatch& b, const float2* x, float2* y, cudaStream_t s) {
  const NufftGeom& g = p->g;
  if (!b.bin) PG_TRY(nufft_plain_binning(p, s));
  const Binning* bin = b.bin ? b.bin : p->plain.get();
  const int L = bin->L;
  const int Cb = batch_coils(p, b.C, L);
  const uint64_t G = g.ngrid();
  for (int c0 = 0; c0 < b.C; c0 += Cb) {
    const int nb = std::min(Cb, b.C - c0);
    const int B = nb * L;
    if (p->own_fft) {
      PG_TRY(ensure_workspace(p, B, nullptr, s));
      PG_TRY(grow(p->work->fin, fftpass_scratch(g, B), s));
      ProfScope ps("fft_fwd", s);
      if (b.cgroup > 0) {
        // one pass per image over its coils of the batch, into their grids
        for (int i0 = c0; i0 < c0 + nb;) {
          const int img = i0 / b.cgroup;
          const int i1 = std::min(c0 + nb, (img + 1) * b.cgroup);
          PG_TRY(fftpass_forward(g, (i1 - i0) * L, L, x + (uint64_t)img * b.image_stride, b.S, i0, b.E,
                                 b.Wo ? b.Wo + (uint64_t)img * b.phase_stride : nullptr, p->deapf.p, p->tw2d.p,
                                 p->work->fin.p, p->work->grids.p + (uint64_t)(i0 - c0) * L * G, s));
          i0 = i1;
        }
      } else {
        PG_TRY(fftpass_forward(g, B, L, x, b.S, c0, b.E, b.Wo, p->deapf.p, p->tw2d.p, p->work->fin.p,
                               p->work->grids.p, s));
      }
    } else {
    cufftHandle h;
    PG_TRY(ensure_workspace(p, B, &h, s));
    PG_TRY(ensure_forward_input(p, B, s));
    {
      ProfScope ps("pre", s);
      if (b.cgroup > 0) {
        for (int i0 = c0; i0 < c0 + nb;) {
          const int img = i0 / b.cgroup;
          const int i1 = std::min(c0 + nb, (img + 1) * b.cgroup);
          PG_LAUNCH_PDL(k_pre, dim3(ceil_div(g.nimg(), 256), (i1 - i0) * L), 256, 0, s, g, L,
                    x + (uint64_t)img * b.image_stride, b.S, i0, b.E,
                    b.Wo ? b.Wo + (uint64_t)img * b.phase_stride : nullptr, p->deapf.p,
                    p->work->fin.p + (uint64_t)(i0 - c0) * L * G);
          i0 = i1;
        }
      } else {
        PG_LAUNCH_PDL(k_pre, dim3(ceil_div(g.nimg(), 256), B), 256, 0, s, g, L, x, b.S, c0, b.E, b.Wo, p->deapf.p,
                  p->work->fin.p);
      }
    }
    {
      ProfScope ps("fft_fwd", s);
      PG_CUFFT(cufftExecC2C(h, reinterpret_cast<cufftComplex*>(p->work->fin.p),
                            reinterpret_cast<cufftComplex*>(p->work->grids.p), CUFFT_FORWARD));
    }
    }
    float2* yc = y + (uint64_t)c0 * b.data_stride;
    const float2* aa = (L > 1 || bin->aa.p) ? bin->aa.p : nullptr;
    ProfScope ps("gather", s);
    if (bin->nsub > 0) PG_TRY(launch_gather(p, bin, aa, nb, yc, b.data_stride, s));
  }
  return PG_OK;
}

pg_status nufft_adjoint(NufftPlan* p, const NufftBatch& b, const float2* y, float2* x, cudaStream_t s) {
  const NufftGeom& g = p->g;
  if (!b.bin) PG_TRY(nufft_plain_binning(p, s));
  const Binning* bin = b.bin ? b.bin : p->plain.get();
  const int L = bin->L, K = bin->K;
  const int Cb = batch_coils(p, b.C, L);
  const uint64_t G = g.ngrid();
  const TileShape& t = bin->tile;
  const size_t plane_bytes = (size_t)t.PX * t.PY * t.PZ * 2 * sizeof(float);
  const size_t smem_limit = (size_t)smem_optin_bytes() - 2048;   // static shared arrays + margin
  const int smax = bin->submax;
  // tile planes of cc coils x K segments, plus the staged samples
  auto smem_for = [&](int cc) {
    return plane_bytes * K * cc + (size_t)smax * (spread_wrow(g.dim) * sizeof(float) + sizeof(uint2) +
                                                  (size_t)K * cc * sizeof(float2));
  };
  // 2-D with K <= 2 (Hanning segments or none): the folded spread reads the
  // data vector itself; otherwise k_adjoint_prep forms the values first.
  const bool folded = (g.dim == 2 && K <= 2 && (t.TX == 16 || t.TX == 32));
  int Cc = std::max(1, std::min(4, p->tune.spread_cc));
  if (folded) {
    Cc = Cc >= 4 ? 4 : Cc >= 2 ? 2 : 1;
    while (Cc > 1 && (Cc >= 2 * std::min(Cb, b.C) || spread2d_smem(t.TX, Cc * K, smax) > smem_limit)) Cc >>= 1;
    if (spread2d_smem(t.TX, K, smax) > smem_limit)
      return set_error(PG_INVALID_ARG, "adjoint: tile of %d cells too large for shared memory", t.TX);
  } else {
    while (Cc > 1 && (Cc * K > 16 || smem_for(Cc) > smem_limit)) --Cc;
    if (K > 16 || smem_for(1) > smem_limit)
      return set_error(PG_INVALID_ARG, "adjoint: segment window K=%d too wide for shared memory", K);
  }
  const float w1 = p->lut_max;
  const float wmax = (g.dim == 2) ? w1 * w1 : w1 * w1 * w1;
  for (int c0 = 0; c0 < b.C; c0 += Cb) {
    const int nb = std::min(Cb, b.C - c0);
    const int B = nb * L;
    cufftHandle h = 0;
    PG_TRY(ensure_workspace(p, B, p->own_fft ? nullptr : &h, s));
    const float2* yc = y + (uint64_t)c0 * b.data_stride;
    const float2* aa = (L > 1 || bin->aa.p) ? bin->aa.p : nullptr;
    // spread target: on the 2-D own FFT passes a grid set kept zero between
    // adjoints (its first inverse pass clears it); else the forward's grids,
    // cleared here
    const bool self_clear = self_clearing(*p);
    float2* target = p->work->grids.p;
    if (self_clear) {
      PG_TRY(ensure_adjoint_grids(p, B, s));
      target = p->work->agrids.p;
    }
    {
    // the adjoint gridding as the reference's gridding_adjoint (gridding.cpp:31-214),
    // timed as one stage (with the grids' clearing where it is a separate step)
    ProfScope pag("adjoint_gridding", s);
    if (folded) {
      if (!self_clear) {
        ProfScope ps("prep", s);
        PG_CUDA(cudaMemsetAsync(target, 0, (size_t)B * G * sizeof(float2), s));
      }
      p->work->agrids_clean = false;
      if (bin->nsub > 0) {
        ProfScope ps("spread", s);
        if (t.TX == 32) PG_TRY(spread2d_launch_t<32>(p, bin, Cc, aa, yc, b.data_stride, nb, wmax, target, s));
        else PG_TRY(spread2d_launch_t<16>(p, bin, Cc, aa, yc, b.data_stride, nb, wmax, target, s));
      }
    } else {
    PG_TRY(grow(p->work->vs, (uint64_t)nb * bin->M * K, s));
    {
      ProfScope ps("prep", s);
      // a self-clearing target is already zero: only the values are formed
      const uint64_t n4 = self_clear ? 0 : (uint64_t)B * G / 2;   // G is even: float2 pairs -> float4 words
      const uint64_t work = std::max<uint64_t>(n4, bin->M);
      PG_LAUNCH(k_adjoint_prep, (unsigned)std::min<uint64_t>(ceil_div(work, 256), 8ull * sm_count()), 256, 0, s, n4,
                reinterpret_cast<float4*>(target), nb, bin->M, K, bin->perm.p, aa, yc, b.data_stride,
                p->work->vs.p);
    }
    p->work->agrids_clean = false;
    if (bin->nsub > 0) {
      ProfScope ps("spread", s);
      // full chunks of cc coils, then the remaining coils in one chunk
      const int cc = std::min(Cc, nb);
      const int full = nb / cc, rest = nb - full * cc;
      SpreadArgs a{p->work->vs.p, 0, cc, full, wmax, smem_for(cc)};
      PG_TRY(launch_spread(p, bin, a, target, s));
      if (rest > 0) {
        SpreadArgs r{p->work->vs.p, full * cc, rest, 1, wmax, smem_for(rest)};
        PG_TRY(launch_spread(p, bin, r, target, s));
      }
    }
    }
    }
    const int acc = (b.accumulate || c0 > 0) ? 1 : 0;
    if (p->own_fft) {
      PG_TRY(grow(p->work->fin, fftpass_scratch(g, B), s));
      PG_TRY(grow(p->work->rimg, (uint64_t)B * g.nimg(), s));
      ProfScope ps("fft_adj", s);
      if (b.cgroup > 0) {
        // one pass per image over its coils of the batch; an image whose
        // coils began in an earlier batch adds to its sum
        for (int i0 = c0; i0 < c0 + nb;) {
          const int img = i0 / b.cgroup;
          const int i1 = std::min(c0 + nb, (img + 1) * b.cgroup);
          const int acc_img = (b.accumulate || i0 > img * b.cgroup) ? 1 : 0;
          PG_TRY(fftpass_adjoint(g, (i1 - i0) * L, L, target + (uint64_t)(i0 - c0) * L * G, self_clear, b.S, i0, b.E,
                                 b.WoH ? b.WoH + (uint64_t)img * b.phase_stride : nullptr, p->deapf.p, p->tw2d.p,
                                 p->work->fin.p, p->work->rimg.p, acc_img, x + (uint64_t)img * b.image_stride, s));
          i0 = i1;
        }
      } else {
        PG_TRY(fftpass_adjoint(g, B, L, target, self_clear, b.S, c0, b.E, b.WoH, p->deapf.p, p->tw2d.p,
                               p->work->fin.p, p->work->rimg.p, acc, x, s));
      }
      if (self_clear) p->work->agrids_clean = true;   // the first inverse pass leaves the target zero
      continue;
    }
    {
      ProfScope ps("fft_adj", s);
      PG_CUFFT(cufftExecC2C(h, reinterpret_cast<cufftComplex*>(p->work->grids.p),
                            reinterpret_cast<cufftComplex*>(p->work->grids.p), CUFFT_INVERSE));
    }
    ProfScope ps("post", s);
    if (b.cgroup > 0) {
      for (int i0 = c0; i0 < c0 + nb;) {
        const int img = i0 / b.cgroup;
        const int i1 = std::min(c0 + nb, (img + 1) * b.cgroup);
        const int acc_img = (b.accumulate || i0 > img * b.cgroup) ? 1 : 0;
        PG_TRY(launch_post(p, i1 - i0, L, b, b.WoH ? b.WoH + (uint64_t)img * b.phase_stride : nullptr,
                           p->work->grids.p + (uint64_t)(i0 - c0) * L * G, i0, acc_img,
                           x + (uint64_t)img * b.image_stride, s));
        i0 = i1;
      }
    } else {
      PG_TRY(launch_post(p, nb, L, b, b.WoH, p->work->grids.p, c0, acc, x, s));
    }
  }
  return PG_OK;
}

}  // namespace pg
