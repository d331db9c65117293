// Exact field-corrected DFT (Gdft) for sm_100a.
//
// Reference: ftCpu / iftCpu (ftCpu.cpp:95-215), called by Gdft (Gdft.cpp:53-136):
//   forward  y_i = sum_j x_j exp(-i (2pi k_i . r_j + FM_j t_i))
//   adjoint  x_j = sum_i y_i exp(+i (2pi k_i . r_j + FM_j t_i))
// The reference evaluates the phase and sinf/cosf in FP32.  Here the phase
// is formed with FP64 products and reduced mod 2pi in FP64, then one FP32
// __sincosf serves every coil of the pair; the complex MACs are FP32 with a
// two-level (per-tile, then running) sum.
//
// GdftR2 (ftCpuWithGrads.cpp:93-216) multiplies each pair by
//   sinc(kx_i/Nx + Gx_j t_i) sinc(ky_i/Ny + Gy_j t_i) sinc(kz_i/Nz + Gz_j t_i),
// sinc(a) = sin(pi a)/(pi a) (1 for |a| < 1e-4), Gx/Gy/Gz the field map's
// differences (GdftR2.cpp:62-110): the same kernels with GRAD = true.
//
// Layout: one thread per output (sample for forward, voxel for adjoint);
// the other side is staged in shared-memory tiles of 128 entries.  Within a
// tile each coil keeps two complex sums, A = sum cos(ph) v and B = sum
// sin(ph) v, each one paired fp32 fma per pair with v as loaded; they are
// combined once per tile (forward A - iB, adjoint A + iB).  When the
// outputs alone do not fill the GPU the inner sum is split over blockIdx.y
// and the partial sums are combined in a fixed order (deterministic).
#include <vector>

#include "pg_gdft.cuh"
#include "pg_profile.cuh"

namespace pg {

namespace {
constexpr int kTile = 128;
constexpr int kCoilChunk = 8;

// sincPG (ftCpuWithGrads.cpp:76-84)
__device__ __forceinline__ float sinc_pg(float a) {
  return fabsf(a) < 0.0001f ? 1.0f : sinpif(a) / (3.14159265358979323846f * a);
}

// The pair's through-voxel dephasing factor: kn = (kx/Nx, ky/Ny, kz/Nz, t),
// gm = (Gx, Gy, Gz, -).
__device__ __forceinline__ float grad_factor(float4 kn, float4 gm) {
  return sinc_pg(kn.x + gm.x * kn.w) * sinc_pg(kn.y + gm.y * kn.w) * sinc_pg(kn.z + gm.z * kn.w);
}

__device__ __forceinline__ void phase_sincos(double ph, float* s, float* c) {
  const double inv2pi = 0.15915494309189533577;   // 1 / (2 pi)
  const double twopi = 6.283185307179586476925;    // 2 pi (double)
  const double n = rint(ph * inv2pi);
  const float r = (float)fma(-n, twopi, ph);      // |r| <= pi
  __sincosf(r, s, c);
}
}  // namespace

// Forward partial sums.  ks[i] = (2pi kx, 2pi ky, 2pi kz, t); vs[j] = (ix, iy, iz, FM).
// xin: nc x ni inputs (already multiplied by the coil maps).
template <int NC, bool GRAD>
__global__ void __launch_bounds__(kTile) k_dft_forward(uint64_t nk, uint64_t ni, const double4* __restrict__ ks,
                                                       const double4* __restrict__ vs,
                                                       const float4* __restrict__ kns, const float4* __restrict__ gms,
                                                       const float2* __restrict__ xin, uint64_t jchunk,
                                                       float2* __restrict__ part) {
  __shared__ double4 sv[kTile];
  __shared__ float2 sx[NC][kTile];
  __shared__ float4 sg[GRAD ? kTile : 1];
  const uint64_t i = (uint64_t)blockIdx.x * kTile + threadIdx.x;
  const uint64_t j0 = (uint64_t)blockIdx.y * jchunk;
  const uint64_t j1 = min(ni, j0 + jchunk);
  double4 k = make_double4(0, 0, 0, 0);
  float4 kn = make_float4(0.f, 0.f, 0.f, 0.f);
  if (i < nk) {
    k = ks[i];
    if (GRAD) kn = kns[i];
  }
  float2 tot[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) tot[c] = make_float2(0.f, 0.f);
  for (uint64_t jt = j0; jt < j1; jt += kTile) {
    const int n = (int)((j1 - jt) < (uint64_t)kTile ? (j1 - jt) : (uint64_t)kTile);
    __syncthreads();
    if (threadIdx.x < n) {
      sv[threadIdx.x] = vs[jt + threadIdx.x];
      if (GRAD) sg[threadIdx.x] = gms[jt + threadIdx.x];
#pragma unroll
      for (int c = 0; c < NC; ++c) sx[c][threadIdx.x] = xin[(uint64_t)c * ni + jt + threadIdx.x];
    }
    __syncthreads();
    float2 acA[NC], acB[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acA[c] = acB[c] = make_float2(0.f, 0.f);
    for (int j = 0; j < n; ++j) {
      const double4 v = sv[j];
      const double ph = fma(k.x, v.x, fma(k.y, v.y, fma(k.z, v.z, v.w * k.w)));
      float s, co;
      phase_sincos(ph, &s, &co);
      if (GRAD) {
        const float b = grad_factor(kn, sg[j]);
        s *= b;
        co *= b;
      }
      const float2 cp = make_float2(co, co), sp = make_float2(s, s);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float2 x = sx[c][j];
        acA[c] = __ffma2_rn(cp, x, acA[c]);
        acB[c] = __ffma2_rn(sp, x, acB[c]);
      }
    }
    // e^{-i ph} x = cos x - i sin x: re += A.x + B.y, im += A.y - B.x
#pragma unroll
    for (int c = 0; c < NC; ++c) { tot[c].x += acA[c].x + acB[c].y; tot[c].y += acA[c].y - acB[c].x; }
  }
  if (i < nk) {
#pragma unroll
    for (int c = 0; c < NC; ++c) part[((uint64_t)blockIdx.y * NC + c) * nk + i] = tot[c];
  }
}

// Adjoint partial sums.  yin: nc x nk data (coil-major, stride dstride).
template <int NC, bool GRAD>
__global__ void __launch_bounds__(kTile) k_dft_adjoint(uint64_t nk, uint64_t ni, const double4* __restrict__ ks,
                                                       const double4* __restrict__ vs,
                                                       const float4* __restrict__ kns, const float4* __restrict__ gms,
                                                       const float2* __restrict__ yin, uint64_t dstride,
                                                       uint64_t ichunk, float2* __restrict__ part) {
  __shared__ double4 sk[kTile];
  __shared__ float2 sy[NC][kTile];
  __shared__ float4 skn[GRAD ? kTile : 1];
  const uint64_t j = (uint64_t)blockIdx.x * kTile + threadIdx.x;
  const uint64_t i0 = (uint64_t)blockIdx.y * ichunk;
  const uint64_t i1 = min(nk, i0 + ichunk);
  double4 v = make_double4(0, 0, 0, 0);
  float4 gm = make_float4(0.f, 0.f, 0.f, 0.f);
  if (j < ni) {
    v = vs[j];
    if (GRAD) gm = gms[j];
  }
  float2 tot[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) tot[c] = make_float2(0.f, 0.f);
  for (uint64_t it = i0; it < i1; it += kTile) {
    const int n = (int)((i1 - it) < (uint64_t)kTile ? (i1 - it) : (uint64_t)kTile);
    __syncthreads();
    if (threadIdx.x < n) {
      sk[threadIdx.x] = ks[it + threadIdx.x];
      if (GRAD) skn[threadIdx.x] = kns[it + threadIdx.x];
#pragma unroll
      for (int c = 0; c < NC; ++c) sy[c][threadIdx.x] = yin[(uint64_t)c * dstride + it + threadIdx.x];
    }
    __syncthreads();
    float2 acA[NC], acB[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acA[c] = acB[c] = make_float2(0.f, 0.f);
    for (int q = 0; q < n; ++q) {
      const double4 k = sk[q];
      const double ph = fma(k.x, v.x, fma(k.y, v.y, fma(k.z, v.z, v.w * k.w)));
      float s, co;
      phase_sincos(ph, &s, &co);
      if (GRAD) {
        const float b = grad_factor(skn[q], gm);
        s *= b;
        co *= b;
      }
      const float2 cp = make_float2(co, co), sp = make_float2(s, s);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const float2 y = sy[c][q];
        acA[c] = __ffma2_rn(cp, y, acA[c]);
        acB[c] = __ffma2_rn(sp, y, acB[c]);
      }
    }
    // e^{+i ph} y = cos y + i sin y: re += A.x - B.y, im += A.y + B.x
#pragma unroll
    for (int c = 0; c < NC; ++c) { tot[c].x += acA[c].x - acB[c].y; tot[c].y += acA[c].y + acB[c].x; }
  }
  if (j < ni) {
#pragma unroll
    for (int c = 0; c < NC; ++c) part[((uint64_t)blockIdx.y * NC + c) * ni + j] = tot[c];
  }
}

// x_c = S_c * x (SENSE.cpp:59-63), for coils [c0, c0+nc).
__global__ void k_apply_maps(uint64_t ni, int nc, int c0, const float2* __restrict__ S, const float2* __restrict__ x,
                             float2* __restrict__ out) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ni) return;
  const float2 xv = x[j];
  for (int c = 0; c < nc; ++c) out[(uint64_t)c * ni + j] = S ? cmul(S[(uint64_t)(c0 + c) * ni + j], xv) : xv;
}

// Forward finalize: y_c[i] = sum over splits (fixed order).
__global__ void k_forward_finish(uint64_t nk, int nc, int nsplit, int ncpad, const float2* __restrict__ part,
                                 float2* __restrict__ y, uint64_t dstride) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nk) return;
  for (int c = 0; c < nc; ++c) {
    float2 s = part[(uint64_t)c * nk + i];
    for (int q = 1; q < nsplit; ++q) s = cadd(s, part[((uint64_t)q * ncpad + c) * nk + i]);
    y[(uint64_t)c * dstride + i] = s;
  }
}

// Adjoint finalize: x_j (+)= sum_c img_c * conj(S_c) (SENSE.cpp:84-96).
__global__ void k_adjoint_finish(uint64_t ni, int nc, int c0, int nsplit, int ncpad, const float2* __restrict__ part,
                                 const float2* __restrict__ S, int accumulate, float2* __restrict__ x) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ni) return;
  float2 acc = accumulate ? x[j] : make_float2(0.f, 0.f);
  for (int c = 0; c < nc; ++c) {
    float2 s = part[(uint64_t)c * ni + j];
    for (int q = 1; q < nsplit; ++q) s = cadd(s, part[((uint64_t)q * ncpad + c) * ni + j]);
    if (S) s = cmul(s, cconj(S[(uint64_t)(c0 + c) * ni + j]));
    acc = (c == 0 && !accumulate) ? s : cadd(acc, s);
  }
  x[j] = acc;
}

static pg_status upload_samples(GdftPlan* p, uint64_t nk, const float* kx, const float* ky, const float* kz,
                                const float* t, cudaStream_t s);

pg_status gdft_plan_create(std::unique_ptr<GdftPlan>* out, uint64_t nk, uint64_t ni, const float* kx, const float* ky,
                           const float* kz, const float* ix, const float* iy, const float* iz, const float* fm,
                           const float* t, cudaStream_t s) {
  if (nk == 0 || ni == 0) return set_error(PG_INVALID_ARG, "Gdft: empty operator");
  auto p = std::make_unique<GdftPlan>();
  p->nk = nk;
  p->ni = ni;
  std::vector<double4> vs(ni);
  for (uint64_t j = 0; j < ni; ++j) {
    if (!(std::isfinite(ix[j]) && std::isfinite(iy[j]) && std::isfinite(iz[j]) && std::isfinite(fm[j])))
      return set_error(PG_INVALID_ARG, "Gdft: non-finite voxel input at %llu", (unsigned long long)j);
    vs[j] = make_double4(ix[j], iy[j], iz[j], fm[j]);
  }
  PG_TRY(p->vs.upload(vs.data(), ni, s));
  PG_TRY(upload_samples(p.get(), nk, kx, ky, kz, t, s));
  *out = std::move(p);
  return PG_OK;
}

static pg_status upload_samples(GdftPlan* p, uint64_t nk, const float* kx, const float* ky, const float* kz,
                                const float* t, cudaStream_t s) {
  const double tpi = 6.283185307179586476925;
  std::vector<double4> ks(nk);
  for (uint64_t i = 0; i < nk; ++i) {
    if (!(std::isfinite(kx[i]) && std::isfinite(ky[i]) && std::isfinite(kz[i]) && std::isfinite(t[i])))
      return set_error(PG_INVALID_ARG, "Gdft: non-finite sample input at %llu", (unsigned long long)i);
    ks[i] = make_double4(tpi * kx[i], tpi * ky[i], tpi * kz[i], (double)t[i]);
  }
  PG_TRY(p->ks.upload(ks.data(), nk, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

pg_status gdft_plan_same_voxels(std::unique_ptr<GdftPlan>* out, const GdftPlan& src, uint64_t nk, const float* kx,
                                const float* ky, const float* kz, const float* t, cudaStream_t s) {
  if (nk == 0) return set_error(PG_INVALID_ARG, "Gdft: empty operator");
  auto p = std::make_unique<GdftPlan>();
  p->nk = nk;
  p->ni = src.ni;
  p->vs.borrow(src.vs);
  p->work = src.work;
  PG_TRY(upload_samples(p.get(), nk, kx, ky, kz, t, s));
  *out = std::move(p);
  return PG_OK;
}

pg_status gdft_plan_add_gradients(GdftPlan* p, const float* kx, const float* ky, const float* kz, const float* t,
                                  const float* fm, int nx, int ny, int nz, cudaStream_t s) {
  const uint64_t N = (uint64_t)nx * ny * nz;
  if (nx < 1 || ny < 1 || nz < 1 || N != p->ni)
    return set_error(PG_INVALID_ARG, "GdftR2: nx*ny*nz = %llu does not match %llu voxels", (unsigned long long)N,
                     (unsigned long long)p->ni);
  // field-map differences along y, x, z (GdftR2.cpp:62-110: central inside,
  // one-sided over the first and last `offset` entries, no division)
  auto cd = [&](uint64_t off, std::vector<float>* out) {
    out->assign(N, 0.f);
    if (off >= N) return;
    for (uint64_t i = off; i < N - off; ++i) (*out)[i] = fm[i + off] - fm[i - off];
    for (uint64_t i = 0; i < off && i < N; ++i) (*out)[i] = fm[i + off] - fm[i];
    for (uint64_t i = N - off; i < N; ++i) (*out)[i] = fm[i] - fm[i - off];
  };
  std::vector<float> gx, gy, gz;
  cd(1, &gx);
  cd((uint64_t)ny, &gy);
  cd((uint64_t)nx * ny, &gz);
  std::vector<float4> gm(N), kn(p->nk);
  for (uint64_t j = 0; j < N; ++j) gm[j] = make_float4(gx[j], gy[j], gz[j], 0.f);
  for (uint64_t i = 0; i < p->nk; ++i)
    kn[i] = make_float4(kx[i] / (float)nx, ky[i] / (float)ny, kz[i] / (float)nz, t[i]);
  PG_TRY(p->gm.upload(gm.data(), N, s));
  PG_TRY(p->kn.upload(kn.data(), p->nk, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

static int splits_for(uint64_t nout, uint64_t ninner) {
  const uint64_t blocks = (nout + kTile - 1) / kTile;
  const uint64_t want = (uint64_t)sm_count() * 8;
  uint64_t ns = (want + blocks - 1) / blocks;
  const uint64_t max_ns = (ninner + kTile - 1) / kTile;
  if (ns > max_ns) ns = max_ns;
  if (ns < 1) ns = 1;
  if (ns > 64) ns = 64;
  return (int)ns;
}

template <int NC>
static pg_status launch_fwd(GdftPlan* p, int nsplit, uint64_t jchunk, const float2* xin, float2* part, cudaStream_t s) {
  dim3 grid(ceil_div(p->nk, kTile), nsplit);
  if (p->kn.p)
    PG_LAUNCH((k_dft_forward<NC, true>), grid, kTile, 0, s, p->nk, p->ni, p->ks.p, p->vs.p, p->kn.p, p->gm.p, xin,
              jchunk, part);
  else
    PG_LAUNCH((k_dft_forward<NC, false>), grid, kTile, 0, s, p->nk, p->ni, p->ks.p, p->vs.p, nullptr, nullptr, xin,
              jchunk, part);
  return PG_OK;
}
template <int NC>
static pg_status launch_adj(GdftPlan* p, int nsplit, uint64_t ichunk, const float2* yin, uint64_t dstride,
                            float2* part, cudaStream_t s) {
  dim3 grid(ceil_div(p->ni, kTile), nsplit);
  if (p->kn.p)
    PG_LAUNCH((k_dft_adjoint<NC, true>), grid, kTile, 0, s, p->nk, p->ni, p->ks.p, p->vs.p, p->kn.p, p->gm.p, yin,
              dstride, ichunk, part);
  else
    PG_LAUNCH((k_dft_adjoint<NC, false>), grid, kTile, 0, s, p->nk, p->ni, p->ks.p, p->vs.p, nullptr, nullptr, yin,
              dstride, ichunk, part);
  return PG_OK;
}

static int pad_coils(int nc) { return nc <= 1 ? 1 : nc <= 2 ? 2 : nc <= 4 ? 4 : 8; }

pg_status gdft_forward(GdftPlan* p, int C, const float2* S, const float2* x, float2* y, uint64_t dstride,
                       cudaStream_t s) {
  const int nsplit = splits_for(p->nk, p->ni);
  uint64_t jchunk = (p->ni + nsplit - 1) / nsplit;
  jchunk = (jchunk + kTile - 1) / kTile * kTile;
  for (int c0 = 0; c0 < C; c0 += kCoilChunk) {
    const int nc = std::min(kCoilChunk, C - c0);
    const int ncp = pad_coils(nc);
    PG_TRY(grow(p->work->xin, (uint64_t)ncp * p->ni, s));
    PG_TRY(grow(p->work->part, (uint64_t)nsplit * ncp * p->nk, s));
    PG_LAUNCH(k_apply_maps, ceil_div(p->ni, 256), 256, 0, s, p->ni, nc, c0, S, x, p->work->xin.p);
    if (ncp > nc) PG_CUDA(cudaMemsetAsync(p->work->xin.p + (uint64_t)nc * p->ni, 0, (ncp - nc) * p->ni * sizeof(float2), s));
    ProfScope ps("dft_fwd", s);
    switch (ncp) {
      case 1: PG_TRY(launch_fwd<1>(p, nsplit, jchunk, p->work->xin.p, p->work->part.p, s)); break;
      case 2: PG_TRY(launch_fwd<2>(p, nsplit, jchunk, p->work->xin.p, p->work->part.p, s)); break;
      case 4: PG_TRY(launch_fwd<4>(p, nsplit, jchunk, p->work->xin.p, p->work->part.p, s)); break;
      default: PG_TRY(launch_fwd<8>(p, nsplit, jchunk, p->work->xin.p, p->work->part.p, s)); break;
    }
    PG_LAUNCH(k_forward_finish, ceil_div(p->nk, 256), 256, 0, s, p->nk, nc, nsplit, ncp, p->work->part.p,
              y + (uint64_t)c0 * dstride, dstride);
  }
  return PG_OK;
}

pg_status gdft_adjoint(GdftPlan* p, int C, const float2* S, const float2* y, uint64_t dstride, float2* x,
                       cudaStream_t s) {
  const int nsplit = splits_for(p->ni, p->nk);
  uint64_t ichunk = (p->nk + nsplit - 1) / nsplit;
  ichunk = (ichunk + kTile - 1) / kTile * kTile;
  for (int c0 = 0; c0 < C; c0 += kCoilChunk) {
    const int nc = std::min(kCoilChunk, C - c0);
    const int ncp = pad_coils(nc);
    PG_TRY(grow(p->work->part, (uint64_t)nsplit * ncp * p->ni, s));
    // Coils past nc read the first coil's data (valid memory); their sums are discarded.
    const float2* yc = y + (uint64_t)c0 * dstride;
    if (ncp > nc) {
      // stage the chunk contiguously so padded coils stay in bounds
      PG_TRY(grow(p->work->xin, (uint64_t)ncp * p->nk, s));
      for (int c = 0; c < ncp; ++c)
        PG_CUDA(cudaMemcpyAsync(p->work->xin.p + (uint64_t)c * p->nk, yc + (uint64_t)std::min(c, nc - 1) * dstride,
                                p->nk * sizeof(float2), cudaMemcpyDeviceToDevice, s));
      yc = p->work->xin.p;
    }
    const uint64_t stride = (ncp > nc) ? p->nk : dstride;
    ProfScope ps("dft_adj", s);
    switch (ncp) {
      case 1: PG_TRY(launch_adj<1>(p, nsplit, ichunk, yc, stride, p->work->part.p, s)); break;
      case 2: PG_TRY(launch_adj<2>(p, nsplit, ichunk, yc, stride, p->work->part.p, s)); break;
      case 4: PG_TRY(launch_adj<4>(p, nsplit, ichunk, yc, stride, p->work->part.p, s)); break;
      default: PG_TRY(launch_adj<8>(p, nsplit, ichunk, yc, stride, p->work->part.p, s)); break;
    }
    PG_LAUNCH(k_adjoint_finish, ceil_div(p->ni, 256), 256, 0, s, p->ni, nc, c0, nsplit, ncp, p->work->part.p, S,
              c0 > 0 ? 1 : 0, x);
  }
  return PG_OK;
}

}  // namespace pg
