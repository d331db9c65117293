// Kaiser-Bessel window arithmetic shared by the gridding kernels.  Every
// step is the reference's float sequence with no contraction
// (gridding.cpp:62-84), so the window bounds and the LUT entry chosen are
// identical to the reference CPU path.
#pragma once

#include "pg_common.cuh"

namespace pg {

// Grid coordinate s = os*(k + N/2) and the clamped window [lo, hi]
// (gridding.cpp:62-73): hi may be < lo for a sample off the grid.
__device__ __forceinline__ float kb_window(float k, int n_img, float os, float kw, int* lo, int* hi) {
  const float s = __fmul_rn(os, __fadd_rn(k, __fdiv_rn((float)n_img, 2.0f)));
  const float half = __fdiv_rn(__fmul_rn(kw, os), 2.0f);
  *lo = (int)fmaxf(0.0f, ceilf(__fsub_rn(s, half)));
  *hi = (int)fminf(__fsub_rn(__fmul_rn(os, (float)n_img), 1.0f), floorf(__fadd_rn(s, half)));
  return s;
}

// Weight of grid cell c for coordinate s: the nearest-lower LUT entry, 0 past
// the table (gridding.cpp:76-84).  kw2 = kw*kw.
__device__ __forceinline__ float kb_weight(float s, int c, float os, float kw2, const float* __restrict__ lut,
                                           int nlut) {
  const float dist = __fdiv_rn(fabsf(__fsub_rn(s, (float)c)), os);
  const int k0 = (int)__fmul_rn(__fdiv_rn(__fmul_rn(__fmul_rn(dist, dist), 4.0f), kw2), (float)nlut);
  return (k0 >= nlut || k0 < 0) ? 0.0f : lut[k0];
}

}  // namespace pg
