// Exact field-corrected DFT (Gdft) on sm_100a.
#pragma once

#include <cmath>
#include <memory>

#include "pg_common.cuh"

namespace pg {

// Staged coil inputs and split partial sums.  Plans applied one after
// another on one stream (the shots of pcSENSE) share a single one.
struct GdftWork {
  DevBuf<float2> xin;
  DevBuf<float2> part;
};

struct GdftPlan {
  uint64_t nk = 0, ni = 0;
  DevBuf<double4> ks;    // per sample (2pi kx, 2pi ky, 2pi kz, t)
  DevBuf<double4> vs;    // per voxel (ix, iy, iz, FM rad/s); may view another plan's
  std::shared_ptr<GdftWork> work = std::make_shared<GdftWork>();
  // GdftR2 only: per sample (kx/Nx, ky/Ny, kz/Nz, t), per voxel (Gx, Gy, Gz, 0)
  DevBuf<float4> kn;
  DevBuf<float4> gm;
};

pg_status gdft_plan_create(std::unique_ptr<GdftPlan>* out, uint64_t nk, uint64_t ni, const float* kx, const float* ky,
                           const float* kz, const float* ix, const float* iy, const float* iz, const float* fm,
                           const float* t, cudaStream_t s);
// A plan for another trajectory (kx, ky, kz, t of nk samples) over src's voxels:
// views src's voxel table and shares its workspace (src must outlive it and
// both run on one stream).
pg_status gdft_plan_same_voxels(std::unique_ptr<GdftPlan>* out, const GdftPlan& src, uint64_t nk, const float* kx,
                                const float* ky, const float* kz, const float* t, cudaStream_t s);
// Turn p into GdftR2 (GdftR2.cpp:32-110): field-map gradient maps of the
// nx x ny x nz image and the per-pair through-voxel sinc factors.
pg_status gdft_plan_add_gradients(GdftPlan* p, const float* kx, const float* ky, const float* kz, const float* t,
                                  const float* fm, int nx, int ny, int nz, cudaStream_t s);
// y_c = G (S_c x) for C coils; S may be null (C = 1).  y coil stride dstride.
pg_status gdft_forward(GdftPlan* p, int C, const float2* S, const float2* x, float2* y, uint64_t dstride,
                       cudaStream_t s);
// x = sum_c conj(S_c) G^H y_c.
pg_status gdft_adjoint(GdftPlan* p, int C, const float2* S, const float2* y, uint64_t dstride, float2* x,
                       cudaStream_t s);

}  // namespace pg
