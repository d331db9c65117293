// Pruned oversampled FFT passes with the NUFFT pre/post kernels fused in
// (pg_fftpass.cu), for 2-D and 3-D grids of 2N per axis with N a power of two
// (16 ... 512).
#pragma once

#include "pg_nufft.cuh"

namespace pg {

bool fftpass_supported(const NufftGeom& g);
// Scratch (complex elements) the passes need for a batch of B grids.
uint64_t fftpass_scratch(const NufftGeom& g, int B);
// Twiddle tables exp(-2 pi i k1 m2 / n) for the in-plane length (and z),
// made in double precision.
pg_status fftpass_twiddles(const NufftGeom& g, DevBuf<float2>* tw, cudaStream_t s);
// B = Cb*L grids (b = c*L + l).  P: fftpass_scratch elements.  grids: B full grids out.
pg_status fftpass_forward(const NufftGeom& g, int B, int L, const float2* x, const float2* S, int c0,
                          const float2* E, const float2* Wo, const float* deapf, const float2* tw, float2* P,
                          float2* grids, cudaStream_t s);
// grids: B full grids in (after the spread); with clear set the first pass
// zeroes every cell after reading it.  Q: fftpass_scratch elements;
// Rimg: B images; x (+)= their sum in a fixed order.
pg_status fftpass_adjoint(const NufftGeom& g, int B, int L, float2* grids, int clear, const float2* S, int c0,
                          const float2* E, const float2* WoH, const float* deapf, const float2* tw, float2* Q,
                          float2* Rimg, int accumulate, float2* x, cudaStream_t s);

}  // namespace pg
