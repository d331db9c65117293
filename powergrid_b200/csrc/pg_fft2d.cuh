// Pruned oversampled 2-D FFT passes with the NUFFT pre/post kernels fused in
// (pg_fft2d.cu), for 2N x 2N grids with N a power of two (32 ... 512).
#pragma once

#include "pg_nufft.cuh"

namespace pg {

bool fft2d_supported(const NufftGeom& g);
// exp(-2 pi i k / n), k < n = Gx, made in double precision.
pg_status fft2d_twiddles(const NufftGeom& g, DevBuf<float2>* tw, cudaStream_t s);
// B = Cb*L grids (b = c*L + l).  P: B*N*Gy complex scratch.  grids: B full grids out.
pg_status fft2d_forward(const NufftGeom& g, int B, int L, const float2* x, const float2* S, int c0, const float2* E,
                        const float2* Wo, const float* deapf, const float2* tw, float2* P, float2* grids,
                        cudaStream_t s);
// grids: B full grids in (after the spread).  Q: B*N*Gy scratch; Rimg: B*N scratch.
pg_status fft2d_adjoint(const NufftGeom& g, int B, int L, const float2* grids, const float2* S, int c0,
                        const float2* E, const float2* WoH, const float* deapf, const float2* tw, float2* Q,
                        float2* Rimg, int accumulate, float2* x, cudaStream_t s);

}  // namespace pg
