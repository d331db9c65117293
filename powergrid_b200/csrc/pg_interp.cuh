// Kaiser-Bessel interpolation between samples and the oversampled grid with
// no FFT around it: Gnufft::forwardSpatialInterp / adjointSpatialInterp
// (Gnufft.cpp:213-337) at any grid oversampling, and what the reference
// builds on them (reconSupport/directRecon.cpp): Pipe-style density
// compensation, per-coil gridded images and the coil-combined image.
#pragma once

#include <memory>

#include "pg_common.cuh"

namespace pg {

// Grid in the reference's own layout (gridding.cpp:66, 103): y fastest,
// index ny + Gy*(nx + Gx*nz), no shifts and no checkerboard.
struct InterpGeom {
  int dim = 2;
  int Nx = 1, Ny = 1, Nz = 1;
  int Gx = 1, Gy = 1, Gz = 1;
  float os = 2.f, kw = 4.f;
  int nlut = 0;
  __host__ __device__ uint64_t ngrid() const { return (uint64_t)Gx * Gy * Gz; }
};

struct InterpPlan {
  InterpGeom g;
  uint64_t M = 0;
  DevBuf<float> kx, ky, kz;    // original order (kz unused in 2-D)
  DevBuf<float> lut;
  int nbx = 1, nby = 1, nbz = 1;   // 16-cell tiles per axis
  DevBuf<uint32_t> perm;       // samples sorted by the tile of their window's low corner
  DevBuf<uint32_t> starts;     // first sorted position per tile
  // adjoint work items (tile, first range, ranges, partial slot or -1), their
  // sorted-sample ranges, and per tile with several items (tile, first slot, slots)
  DevBuf<int4> items;
  DevBuf<uint2> segs;
  DevBuf<int4> fix;
  int nitems = 0, nfix = 0, nslots = 0;
  DevBuf<float2> partial;      // partial tiles of the further items
  DevBuf<float2> tmp;          // density compensation: samples
  DevBuf<float2> grid;         // density compensation: grid
};

// Tables for M samples on a (gridos * N)^d grid; k in cycles/FOV as Gnufft
// takes them.  Grid sizes follow Gnufft.cpp:55-61 and 221-229 (the element
// count must equal Gx*Gy*Gz, i.e. gridos*N integral and even in-plane).
// unit_peak divides the LUT by its first entry (density compensation only).
pg_status interp_plan_create(std::unique_ptr<InterpPlan>* out, uint64_t M, float gridos, int nx, int ny, int nz,
                             const float* kx, const float* ky, const float* kz, cudaStream_t s,
                             bool unit_peak = false);
// y[i] = sum over the clamped window of w * grid (gridding.cpp:217-415).
pg_status interp_forward(const InterpPlan* p, const float2* grid, float2* y, cudaStream_t s);
// grid = sum over samples of w * d (gridding.cpp:31-214); every cell written.
pg_status interp_adjoint(const InterpPlan* p, const float2* d, float2* grid, cudaStream_t s);
// calc3DDensityCompensation (directRecon.cpp:28-61) on p (built at gridos 3
// with unit_peak by the caller): |dcf| / ||dcf||_2 after two iterations of
// dcf <- dcf / Re(interp(interp^H(dcf))).
pg_status density_compensation(InterpPlan* p, float* dcf, cudaStream_t s);

}  // namespace pg
