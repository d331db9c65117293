// Spatial interpolation with no FFT around it (Gnufft::forwardSpatialInterp /
// adjointSpatialInterp, Gnufft.cpp:213-337), density compensation
// (reconSupport/directRecon.cpp:28-61), per-coil gridded images
// (directRecon.cpp:108-133) and the coil-combined image (directRecon.cpp:63-73).
//
// The grids here are the reference's own (unshifted, y fastest) and the
// oversampling is any factor up to 3.75 (16 taps per axis), so these kernels
// take the window bounds per sample instead of the fixed 8 taps of the
// operator path.
//   forward: one warp per sample; the per-axis window weights are computed
//            once (lane a: cell a of each axis) and shuffled; half-warps walk
//            alternate (z, x) rows with lane & 15 on the y cell, so a half
//            warp reads one grid column; butterfly sum.
//   adjoint: gather form, no atomics.  Samples are sorted (device counting
//            sort, stable) by the 16-cell tile holding their window's low
//            corner; the samples that can reach an output tile are those of
//            its own bin and the previous bin along each axis (a window spans
//            at most 16 cells).  They are cut into work items of at most 512
//            samples; a block takes one item, stages its samples in shared
//            memory and sums them into the tile's cells in registers.  A
//            tile's first item stores the cells (so no zeroing pass is
//            needed), further items store partial tiles that a second kernel
//            adds in item order: every cell's sum has a fixed order.
#include <algorithm>
#include <cmath>
#include <vector>

#include "pg_binsort.cuh"
#include "pg_interp.cuh"
#include "pg_kb.cuh"
#include "pg_nufft.cuh"
#include "pg_ops.cuh"

namespace pg {
namespace {

constexpr int kTileI = 16;     // adjoint tile edge (cells)
constexpr int kMaxTaps = 16;   // cells per axis in one window
constexpr int kChunk = 128;    // samples staged per round
constexpr uint32_t kItemSamples = 512;  // samples per adjoint work item

__global__ void k_interp_forward(InterpGeom g, uint64_t M, const float* __restrict__ kx, const float* __restrict__ ky,
                                 const float* __restrict__ kz, const float* __restrict__ lut,
                                 const float2* __restrict__ grid, float2* __restrict__ y) {
  const uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (i >= M) return;  // warp-uniform
  const float kw2 = __fmul_rn(g.kw, g.kw);
  int xl, xh, yl, yh, zl = 0, zh = 0;
  const float sx = kb_window(kx[i], g.Nx, g.os, g.kw, &xl, &xh);
  const float sy = kb_window(ky[i], g.Ny, g.os, g.kw, &yl, &yh);
  float sz = 0.f;
  if (g.dim == 3) sz = kb_window(kz[i], g.Nz, g.os, g.kw, &zl, &zh);
  const int nxT = max(0, xh - xl + 1), nyT = max(0, yh - yl + 1), nzT = max(0, zh - zl + 1);
  // lane a holds the weights of window cell a along each axis
  const float wxl = lane < nxT ? kb_weight(sx, xl + lane, g.os, kw2, lut, g.nlut) : 0.f;
  const float wyl = lane < nyT ? kb_weight(sy, yl + lane, g.os, kw2, lut, g.nlut) : 0.f;
  const float wzl = (g.dim == 3 && lane < nzT) ? kb_weight(sz, zl + lane, g.os, kw2, lut, g.nlut) : 0.f;
  // half-warps take alternate (z, x) rows; lane & 15 is the y cell
  const int ly = lane & 15;
  const float wy = __shfl_sync(0xffffffffu, wyl, ly);
  const int rows = nxT * nzT;
  int ix = lane >> 4, iz = 0;
  while (nxT > 0 && ix >= nxT) { ix -= nxT; ++iz; }
  float ar = 0.f, ai = 0.f;
  for (int r0 = 0; r0 < rows; r0 += 2) {  // warp-uniform trip count
    const bool row_ok = r0 + (lane >> 4) < rows;
    const float wx = __shfl_sync(0xffffffffu, wxl, row_ok ? ix : 0);
    const float wz = __shfl_sync(0xffffffffu, wzl, row_ok ? iz : 0);
    if (row_ok && ly < nyT) {
      // w = kbX * kbY (* kbZ) as gridding.cpp:63, 100
      float w = __fmul_rn(wx, wy);
      if (g.dim == 3) w = __fmul_rn(w, wz);
      const float2 v =
          grid[(uint64_t)(yl + ly) + (uint64_t)g.Gy * ((uint64_t)(xl + ix) + (uint64_t)g.Gx * (uint64_t)(zl + iz))];
      ar = __fadd_rn(ar, __fmul_rn(w, v.x));
      ai = __fadd_rn(ai, __fmul_rn(w, v.y));
    }
    ix += 2;
    while (nxT > 0 && ix >= nxT) { ix -= nxT; ++iz; }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    ar = __fadd_rn(ar, __shfl_xor_sync(0xffffffffu, ar, o));
    ai = __fadd_rn(ai, __shfl_xor_sync(0xffffffffu, ai, o));
  }
  if (lane == 0) y[i] = make_float2(ar, ai);
}

// Bin key: the tile of the window's low corner (clamped to the last tile for
// samples whose window lies past the grid edge; they touch no cell).
__global__ void k_interp_keys(InterpGeom g, uint64_t M, const float* __restrict__ kx, const float* __restrict__ ky,
                              const float* __restrict__ kz, int nbx, int nby, int nbz, uint32_t* __restrict__ key) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  int xl, xh, yl, yh, zl = 0, zh = 0;
  kb_window(kx[i], g.Nx, g.os, g.kw, &xl, &xh);
  kb_window(ky[i], g.Ny, g.os, g.kw, &yl, &yh);
  if (g.dim == 3) kb_window(kz[i], g.Nz, g.os, g.kw, &zl, &zh);
  const int bx = min(xl / kTileI, nbx - 1), by = min(yl / kTileI, nby - 1), bz = min(zl / kTileI, nbz - 1);
  key[i] = (uint32_t)(((uint64_t)bz * nbx + bx) * nby + by);
}

// One block per work item: a piece (at most kItemSamples samples, in one or
// more sorted ranges) of the samples that reach one output tile (16 x 16
// cells, x 16 z-planes in 3-D: TZ).  A tile's first item stores the grid
// cells; its further items store partial tiles that k_interp_fixup adds in
// item order.
template <int TZ>
__global__ void __launch_bounds__(256) k_interp_adjoint(InterpGeom g, const float* __restrict__ kx,
                                                        const float* __restrict__ ky, const float* __restrict__ kz,
                                                        const float* __restrict__ lut, const float2* __restrict__ d,
                                                        const uint32_t* __restrict__ perm,
                                                        const int4* __restrict__ items, const uint2* __restrict__ segs,
                                                        int nbx, int nby, float2* __restrict__ grid,
                                                        float2* __restrict__ partial) {
  // weights [axis][sample][tap], tap stride 17: a warp's 16 y-cells read 16 banks
  __shared__ float s_w[3][kChunk][kMaxTaps + 1];
  __shared__ int s_lo[3][kChunk];
  __shared__ int s_n[3][kChunk];
  __shared__ float2 s_v[kChunk];
  const int4 it = items[blockIdx.x];   // (tile, first segment, segments, partial slot or -1)
  const int by = it.x % nby;
  const int bx = (it.x / nby) % nbx;
  const int bz = it.x / (nby * nbx);
  const int gy = by * kTileI + (threadIdx.x & 15);
  const int gx = bx * kTileI + (threadIdx.x >> 4);
  const int gz0 = bz * TZ;
  const float kw2 = __fmul_rn(g.kw, g.kw);
  float2 acc[TZ];
#pragma unroll
  for (int z = 0; z < TZ; ++z) acc[z] = make_float2(0.f, 0.f);
  for (int sg = 0; sg < it.z; ++sg) {
    const uint2 seg = segs[it.y + sg];
    for (uint32_t c0 = seg.x; c0 < seg.y; c0 += kChunk) {
      const int cn = (int)min((uint32_t)kChunk, seg.y - c0);
      __syncthreads();  // the previous round is consumed
      if ((int)threadIdx.x < cn) {
        const int q = threadIdx.x;
        const uint32_t j = perm[c0 + q];
        const float kk[3] = {kx[j], ky[j], g.dim == 3 ? kz[j] : 0.f};
        const int nn[3] = {g.Nx, g.Ny, g.Nz};
        for (int a = 0; a < (g.dim == 3 ? 3 : 2); ++a) {
          int lo, hi;
          const float sa = kb_window(kk[a], nn[a], g.os, g.kw, &lo, &hi);
          const int n = max(0, hi - lo + 1);
          s_lo[a][q] = lo;
          s_n[a][q] = n;
          for (int t = 0; t < n; ++t) s_w[a][q][t] = kb_weight(sa, lo + t, g.os, kw2, lut, g.nlut);
        }
        s_v[q] = d[j];
      }
      __syncthreads();
      for (int q = 0; q < cn; ++q) {
        const unsigned dx = (unsigned)(gx - s_lo[0][q]);
        const unsigned dy = (unsigned)(gy - s_lo[1][q]);
        if (dx < (unsigned)s_n[0][q] && dy < (unsigned)s_n[1][q]) {
          const float wxy = __fmul_rn(s_w[0][q][dx], s_w[1][q][dy]);
          const float2 v = s_v[q];
          if (TZ == 1) {
            acc[0].x = __fadd_rn(acc[0].x, __fmul_rn(wxy, v.x));
            acc[0].y = __fadd_rn(acc[0].y, __fmul_rn(wxy, v.y));
          } else {
            const int lz = s_lo[2][q];
            const unsigned nz = (unsigned)s_n[2][q];
#pragma unroll
            for (int z = 0; z < TZ; ++z) {
              const unsigned dz = (unsigned)(gz0 + z - lz);
              if (dz < nz) {
                const float w = __fmul_rn(wxy, s_w[2][q][dz]);
                acc[z].x = __fadd_rn(acc[z].x, __fmul_rn(w, v.x));
                acc[z].y = __fadd_rn(acc[z].y, __fmul_rn(w, v.y));
              }
            }
          }
        }
      }
    }
  }
  if (it.w >= 0) {
    float2* dst = partial + (uint64_t)it.w * (256 * TZ);
#pragma unroll
    for (int z = 0; z < TZ; ++z) dst[z * 256 + threadIdx.x] = acc[z];
    return;
  }
  if (gx >= g.Gx || gy >= g.Gy) return;
#pragma unroll
  for (int z = 0; z < TZ; ++z) {
    const int gz = gz0 + z;
    if (gz < g.Gz) grid[(uint64_t)gy + (uint64_t)g.Gy * ((uint64_t)gx + (uint64_t)g.Gx * gz)] = acc[z];
  }
}

// grid cell += the tile's partials in item order.  fix = (tile, first slot, slots).
template <int TZ>
__global__ void __launch_bounds__(256) k_interp_fixup(InterpGeom g, const int4* __restrict__ fix, int nbx, int nby,
                                                      const float2* __restrict__ partial, float2* __restrict__ grid) {
  const int4 f = fix[blockIdx.x];
  const int by = f.x % nby;
  const int bx = (f.x / nby) % nbx;
  const int bz = f.x / (nby * nbx);
  const int gy = by * kTileI + (threadIdx.x & 15);
  const int gx = bx * kTileI + (threadIdx.x >> 4);
  if (gx >= g.Gx || gy >= g.Gy) return;
  for (int z = 0; z < TZ; ++z) {
    const int gz = bz * TZ + z;
    if (gz >= g.Gz) break;
    const uint64_t cell = (uint64_t)gy + (uint64_t)g.Gy * ((uint64_t)gx + (uint64_t)g.Gx * gz);
    float2 v = grid[cell];
    for (int k = 0; k < f.z; ++k) {
      const float2 q = partial[(uint64_t)(f.y + k) * (256 * TZ) + z * 256 + threadIdx.x];
      v.x = __fadd_rn(v.x, q.x);
      v.y = __fadd_rn(v.y, q.y);
    }
    grid[cell] = v;
  }
}

__global__ void k_fill(uint64_t n, float2 v, float2* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}

// dcf <- dcf / Re(c2) (directRecon.cpp:53)
__global__ void k_div_real(uint64_t n, float2* __restrict__ dcf, const float2* __restrict__ c2) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float r = c2[i].x;
  const float2 v = dcf[i];
  dcf[i] = make_float2(__fdiv_rn(v.x, r), __fdiv_rn(v.y, r));
}

// ||dcf||_2 in FP64: one block, fixed order.
__global__ void __launch_bounds__(1024) k_norm2(uint64_t n, const float2* __restrict__ v, double* __restrict__ out) {
  __shared__ double red[1024];
  double a = 0.0;
  for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double x = v[i].x, y = v[i].y;
    a += x * x + y * y;
  }
  red[threadIdx.x] = a;
  __syncthreads();
  for (int h = blockDim.x / 2; h; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sqrt(red[0]);
}

// |dcf / ||dcf|| |  (directRecon.cpp:57-59)
__global__ void k_abs_scaled(uint64_t n, const float2* __restrict__ v, const double* __restrict__ nrm,
                             float* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float s = (float)*nrm;
  const float2 a = v[i];
  out[i] = (s > 0.f) ? hypotf(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s)) : hypotf(a.x, a.y);
}

// data_c * dcf for one coil (the operand of G / (dcf % data), directRecon.cpp:125)
__global__ void k_scale_real(uint64_t n, const float* __restrict__ w, const float2* __restrict__ x,
                             float2* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_float2(__fmul_rn(w[i], x[i].x), __fmul_rn(w[i], x[i].y));
}

// sqrt(sum_c |img_c|), the coil order fixed (directRecon.cpp:68-70: the sum is
// of magnitudes, not of squared magnitudes).
__global__ void k_sum_magnitudes(uint64_t n, int nc, const float2* __restrict__ img, float* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float acc = 0.f;
  for (int c = 0; c < nc; ++c) {
    const float2 v = img[(uint64_t)c * n + i];
    acc = __fadd_rn(acc, hypotf(v.x, v.y));
  }
  out[i] = sqrtf(acc);
}

pg_status check_trajectory(uint64_t M, int nx, int ny, int nz, const float* kx, const float* ky, const float* kz) {
  for (uint64_t i = 0; i < M; ++i) {
    const float a = kx[i], b = ky[i], c = kz ? kz[i] : 0.f;
    if (!(std::isfinite(a) && std::isfinite(b) && std::isfinite(c)))
      return set_error(PG_INVALID_ARG, "interpolation: non-finite k-space coordinate at %llu", (unsigned long long)i);
    if (std::abs(a) > (nx / 2.0f) * 1.05f || std::abs(b) > (ny / 2.0f) * 1.05f ||
        (nz > 1 && std::abs(c) > (nz / 2.0f) * 1.05f))
      return set_error(PG_INVALID_ARG, "interpolation: k-space trajectory out of range [-N/2, N/2] at %llu",
                       (unsigned long long)i);
  }
  return PG_OK;
}

}  // namespace

// Tables over device coordinates (borrowed; they must outlive the plan).
static pg_status interp_plan_build(InterpPlan* p, cudaStream_t s) {
  const InterpGeom& g = p->g;
  p->nbx = (int)ceil_div((uint64_t)g.Gx, kTileI);
  p->nby = (int)ceil_div((uint64_t)g.Gy, kTileI);
  p->nbz = (g.dim == 3) ? (int)ceil_div((uint64_t)g.Gz, kTileI) : 1;
  const uint64_t nkeys = (uint64_t)p->nbx * p->nby * p->nbz;
  DevBuf<uint32_t> keys;
  PG_TRY(keys.alloc(p->M));
  PG_TRY(p->perm.alloc(p->M));
  PG_TRY(p->starts.alloc(nkeys));
  PG_LAUNCH(k_interp_keys, ceil_div(p->M, 256), 256, 0, s, g, p->M, p->kx.p, p->ky.p, p->kz.p, p->nbx, p->nby,
            p->nbz, keys.p);
  PG_TRY(bin_sort(keys.p, p->M, nkeys, p->perm.p, p->starts.p, s));
  std::vector<uint32_t> st(nkeys);
  PG_CUDA(cudaMemcpyAsync(st.data(), p->starts.p, nkeys * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));  // keys is released on return
  // Work items: per output tile the sorted ranges of the bins that reach it
  // (the tile's own and the previous one along each axis), cut into pieces
  // of at most kItemSamples samples so that dense k-space centres do not
  // serialise in one block.
  std::vector<int4> items, fix;
  std::vector<uint2> segs;
  int slots = 0;
  for (int bz = 0; bz < p->nbz; ++bz)
    for (int bx = 0; bx < p->nbx; ++bx)
      for (int by = 0; by < p->nby; ++by) {
        const int tile = (bz * p->nbx + bx) * p->nby + by;
        const int first_item = (int)items.size();
        int4 cur = make_int4(tile, (int)segs.size(), 0, -1);
        uint32_t fill = 0;
        for (int dzb = (g.dim == 3 ? -1 : 0); dzb <= 0; ++dzb)
          for (int dxb = -1; dxb <= 0; ++dxb)
            for (int dyb = -1; dyb <= 0; ++dyb) {
              const int kbx = bx + dxb, kby = by + dyb, kbz = bz + dzb;
              if (kbx < 0 || kby < 0 || kbz < 0) continue;
              const uint64_t key = ((uint64_t)kbz * p->nbx + kbx) * p->nby + kby;
              uint32_t b0 = st[key];
              const uint32_t b1 = (key + 1 < nkeys) ? st[key + 1] : (uint32_t)p->M;
              while (b0 < b1) {
                if (fill == kItemSamples) {  // close the item, open the next (a partial slot)
                  items.push_back(cur);
                  cur = make_int4(tile, (int)segs.size(), 0, slots++);
                  fill = 0;
                }
                const uint32_t take = std::min(b1 - b0, kItemSamples - fill);
                segs.push_back(make_uint2(b0, b0 + take));
                cur.z += 1;
                fill += take;
                b0 += take;
              }
            }
        items.push_back(cur);
        const int extra = (int)items.size() - first_item - 1;
        if (extra > 0) fix.push_back(make_int4(tile, items[first_item + 1].w, extra, 0));
      }
  p->nitems = (int)items.size();
  p->nfix = (int)fix.size();
  p->nslots = slots;
  PG_TRY(p->items.upload(items.data(), items.size(), s));
  PG_TRY(p->segs.upload(segs.data(), std::max<size_t>(1, segs.size()), s));
  if (!fix.empty()) PG_TRY(p->fix.upload(fix.data(), fix.size(), s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

static pg_status interp_geometry(InterpGeom* g, uint64_t M, float gridos, int nx, int ny, int nz) {
  if (M == 0 || nx < 1 || ny < 1 || nz < 1) return set_error(PG_INVALID_ARG, "interpolation: empty geometry");
  if (M >= (1ull << 32)) return set_error(PG_INVALID_ARG, "interpolation: too many samples");
  if (!(gridos >= 1.0f) || !std::isfinite(gridos))
    return set_error(PG_INVALID_ARG, "interpolation: grid oversampling must be >= 1");
  g->dim = (nz == 1) ? 2 : 3;
  g->Nx = nx; g->Ny = ny; g->Nz = nz;
  g->os = gridos;
  g->kw = 4.0f;  // Gnufft.cpp:84
  if ((int)std::floor(g->kw * gridos) + 1 > kMaxTaps)
    return set_error(PG_INVALID_ARG, "interpolation: gridos %g needs more than %d taps per axis", gridos, kMaxTaps);
  // Gnufft.cpp:221-229
  g->Gx = (int)std::ceil(gridos * (float)nx);
  g->Gy = (int)std::ceil(gridos * (float)ny);
  if (g->Gx % 2) g->Gx += 1;
  if (g->Gy % 2) g->Gy += 1;
  g->Gz = (nz == 1) ? nz : (int)std::ceil(gridos * (float)nz);
  // the reference's grid buffer holds gridOS*Nx*gridOS*Ny(*gridOS*Nz) cells
  // (Gnufft.cpp:56-61); gridding indexes it with gridSize, so the two agree
  // only when gridos*N is an even integer in-plane
  float cells = gridos * (float)nx * gridos * (float)ny;
  if (nz > 1) cells = cells * gridos * (float)nz;
  if ((uint64_t)cells != g->ngrid())
    return set_error(PG_INVALID_ARG, "interpolation: grid of %llu cells does not match gridding's %dx%dx%d",
                     (unsigned long long)(uint64_t)cells, g->Gx, g->Gy, g->Gz);
  return PG_OK;
}

pg_status interp_plan_create(std::unique_ptr<InterpPlan>* out, uint64_t M, float gridos, int nx, int ny, int nz,
                             const float* kx, const float* ky, const float* kz, cudaStream_t s, bool unit_peak) {
  if (!kx || !ky || (nz > 1 && !kz)) return set_error(PG_INVALID_ARG, "interpolation: null argument");
  auto p = std::make_unique<InterpPlan>();
  PG_TRY(interp_geometry(&p->g, M, gridos, nx, ny, nz));
  PG_TRY(check_trajectory(M, nx, ny, nz, kx, ky, nz > 1 ? kz : nullptr));
  p->M = M;
  std::vector<float> lut;
  float beta = 0.f;
  kb_table(gridos, &lut, &beta);
  if (unit_peak) {
    const float peak = lut[0];
    for (auto& v : lut) v = v / peak;
  }
  p->g.nlut = (int)lut.size();
  PG_TRY(p->lut.upload(lut.data(), lut.size(), s));
  PG_TRY(p->kx.upload(kx, M, s));
  PG_TRY(p->ky.upload(ky, M, s));
  if (nz > 1) PG_TRY(p->kz.upload(kz, M, s));
  PG_TRY(interp_plan_build(p.get(), s));
  *out = std::move(p);
  return PG_OK;
}

// A plan over a Gnufft plan's device coordinates (already validated).
static pg_status interp_plan_from_nufft(std::unique_ptr<InterpPlan>* out, const NufftPlan& np, cudaStream_t s) {
  auto p = std::make_unique<InterpPlan>();
  PG_TRY(interp_geometry(&p->g, np.M, np.g.os, np.g.Nx, np.g.Ny, np.g.Nz));
  p->M = np.M;
  std::vector<float> lut;
  float beta = 0.f;
  kb_table(np.g.os, &lut, &beta);
  p->g.nlut = (int)lut.size();
  PG_TRY(p->lut.upload(lut.data(), lut.size(), s));
  p->kx.borrow(np.kx);
  p->ky.borrow(np.ky);
  if (np.g.dim == 3) p->kz.borrow(np.kz);
  PG_TRY(interp_plan_build(p.get(), s));
  *out = std::move(p);
  return PG_OK;
}

pg_status interp_forward(const InterpPlan* p, const float2* grid, float2* y, cudaStream_t s) {
  PG_LAUNCH(k_interp_forward, ceil_div(p->M * 32, 256), 256, 0, s, p->g, p->M, p->kx.p, p->ky.p, p->kz.p, p->lut.p,
            grid, y);
  return PG_OK;
}

pg_status interp_adjoint(const InterpPlan* p, const float2* d, float2* grid, cudaStream_t s) {
  const int tz = p->g.dim == 3 ? kTileI : 1;
  float2* partial = nullptr;
  if (p->nslots > 0) {
    PG_TRY(grow(const_cast<InterpPlan*>(p)->partial, (uint64_t)p->nslots * 256 * tz, s));
    partial = p->partial.p;
  }
  if (p->g.dim == 3) {
    PG_LAUNCH(k_interp_adjoint<kTileI>, p->nitems, 256, 0, s, p->g, p->kx.p, p->ky.p, p->kz.p, p->lut.p, d, p->perm.p,
              p->items.p, p->segs.p, p->nbx, p->nby, grid, partial);
    if (p->nfix) PG_LAUNCH(k_interp_fixup<kTileI>, p->nfix, 256, 0, s, p->g, p->fix.p, p->nbx, p->nby, partial, grid);
  } else {
    PG_LAUNCH(k_interp_adjoint<1>, p->nitems, 256, 0, s, p->g, p->kx.p, p->ky.p, p->kz.p, p->lut.p, d, p->perm.p,
              p->items.p, p->segs.p, p->nbx, p->nby, grid, partial);
    if (p->nfix) PG_LAUNCH(k_interp_fixup<1>, p->nfix, 256, 0, s, p->g, p->fix.p, p->nbx, p->nby, partial, grid);
  }
  return PG_OK;
}

pg_status density_compensation(InterpPlan* p, float* dcf, cudaStream_t s) {
  const uint64_t M = p->M;
  PG_TRY(grow(p->tmp, 2 * M, s));
  PG_TRY(grow(p->grid, p->g.ngrid(), s));
  float2* w = p->tmp.p;        // dcf (complex, as the reference keeps it)
  float2* c2 = p->tmp.p + M;
  // The reference starts from ones / (n * n) (directRecon.cpp:38-40) with the
  // LUT as Gnufft builds it.  The update dcf / Re(F F^H dcf) does not depend
  // on the scale of dcf, scales with the weights' scale squared, and the
  // result is normalised, so the returned dcf does not depend on either
  // scale; the plan's LUT is divided by its peak and dcf starts at 1, which
  // keeps FP32 in range where the reference's float instantiation overflows
  // (peak weight 2.3e7 per axis at gridos 3: 1.2e22 per 3-D tap).
  PG_LAUNCH(k_fill, ceil_div(M, 256), 256, 0, s, M, make_float2(1.0f, 0.f), w);
  for (int it = 0; it < 2; ++it) {  // Niter = 2 (:30), loop :49-55
    PG_TRY(interp_adjoint(p, w, p->grid.p, s));
    PG_TRY(interp_forward(p, p->grid.p, c2, s));
    PG_LAUNCH(k_div_real, ceil_div(M, 256), 256, 0, s, M, w, c2);
  }
  DevBuf<double> nrm;
  PG_TRY(nrm.alloc(1));
  PG_LAUNCH(k_norm2, 1, 1024, 0, s, M, w, nrm.p);
  PG_LAUNCH(k_abs_scaled, ceil_div(M, 256), 256, 0, s, M, w, nrm.p, dcf);
  PG_CUDA(cudaStreamSynchronize(s));  // nrm is released on return
  return PG_OK;
}

// Spatial-interpolation tables of a Gnufft operator: built at construction
// for gridos != 2, on first use otherwise.
static pg_status gnufft_interp(pg_op G, InterpPlan** out, cudaStream_t s) {
  if (!G || G->kind != PG_OP_GNUFFT) return set_error(PG_INVALID_ARG, "spatial interpolation needs a Gnufft operator");
  auto* op = static_cast<GnufftOp*>(G);
  if (!op->interp) PG_TRY(interp_plan_from_nufft(&op->interp, *op->plan, s));
  *out = op->interp.get();
  return PG_OK;
}

}  // namespace pg

using namespace pg;

extern "C" {

pg_status pg_gnufft_grid_length(pg_op G, uint64_t* n) {
  if (!n) return set_error(PG_INVALID_ARG, "null argument");
  PG_TRY(ensure_init());
  InterpPlan* p = nullptr;
  PG_TRY(gnufft_interp(G, &p, default_stream()));
  *n = p->g.ngrid();
  return PG_OK;
}

pg_status pg_gnufft_forward_spatial_interp_device(pg_op G, const void* grid, void* samples, void* stream) {
  if (!grid || !samples) return set_error(PG_INVALID_ARG, "null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  InterpPlan* p = nullptr;
  PG_TRY(gnufft_interp(G, &p, s));
  return interp_forward(p, (const float2*)grid, (float2*)samples, s);
}

pg_status pg_gnufft_adjoint_spatial_interp_device(pg_op G, const void* samples, void* grid, void* stream) {
  if (!grid || !samples) return set_error(PG_INVALID_ARG, "null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  InterpPlan* p = nullptr;
  PG_TRY(gnufft_interp(G, &p, s));
  return interp_adjoint(p, (const float2*)samples, (float2*)grid, s);
}

pg_status pg_gnufft_forward_spatial_interp(pg_op G, const float* grid, float* samples) {
  if (!grid || !samples) return set_error(PG_INVALID_ARG, "null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  InterpPlan* p = nullptr;
  PG_TRY(gnufft_interp(G, &p, s));
  DevBuf<float2> dg, dy;
  PG_TRY(dg.upload((const float2*)grid, p->g.ngrid(), s));
  PG_TRY(dy.alloc(p->M));
  PG_TRY(interp_forward(p, dg.p, dy.p, s));
  PG_CUDA(cudaMemcpyAsync(samples, dy.p, p->M * sizeof(float2), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

pg_status pg_gnufft_adjoint_spatial_interp(pg_op G, const float* samples, float* grid) {
  if (!grid || !samples) return set_error(PG_INVALID_ARG, "null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  InterpPlan* p = nullptr;
  PG_TRY(gnufft_interp(G, &p, s));
  DevBuf<float2> dd, dg;
  PG_TRY(dd.upload((const float2*)samples, p->M, s));
  PG_TRY(dg.alloc(p->g.ngrid()));
  PG_TRY(interp_adjoint(p, dd.p, dg.p, s));
  PG_CUDA(cudaMemcpyAsync(grid, dg.p, p->g.ngrid() * sizeof(float2), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

pg_status pg_density_compensation(const float* kx, const float* ky, const float* kz, uint64_t n, uint64_t n_inplane,
                                  uint64_t nz, float* dcf) {
  if (!kx || !ky || !kz || !dcf) return set_error(PG_INVALID_ARG, "density compensation: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  // Gnufft<T> G(n, overSampling = 3, Ninplane, Ninplane, Nz, ...) (directRecon.cpp:31-35)
  std::unique_ptr<InterpPlan> p;
  PG_TRY(interp_plan_create(&p, n, 3.0f, (int)n_inplane, (int)n_inplane, (int)nz, kx, ky, kz, s, true));
  DevBuf<float> out;
  PG_TRY(out.alloc(n));
  PG_TRY(density_compensation(p.get(), out.p, s));
  PG_CUDA(cudaMemcpyAsync(dcf, out.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

pg_status pg_grid_coil_images(pg_op G, const float* dcf, const float* data, uint64_t nc, float* images) {
  if (!G || !dcf || !data || !images || nc == 0) return set_error(PG_INVALID_ARG, "coil images: bad argument");
  if (G->kind != PG_OP_GNUFFT) return set_error(PG_INVALID_ARG, "coil images need a Gnufft operator");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  const uint64_t M = G->n_data, N = G->n_image;
  DevBuf<float> w;
  DevBuf<float2> d, tmp, img;
  PG_TRY(w.upload(dcf, M, s));
  PG_TRY(d.upload((const float2*)data, M * nc, s));
  PG_TRY(tmp.alloc(M));
  PG_TRY(img.alloc(N * nc));
  for (uint64_t c = 0; c < nc; ++c) {
    PG_LAUNCH(k_scale_real, ceil_div(M, 256), 256, 0, s, M, w.p, d.p + c * M, tmp.p);
    PG_TRY(G->adjoint(tmp.p, img.p + c * N, s));
  }
  PG_CUDA(cudaMemcpyAsync(images, img.p, N * nc * sizeof(float2), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

pg_status pg_sum_of_squares_image(const float* coil_images, uint64_t n, uint64_t nc, float* out) {
  if (!coil_images || !out || n == 0 || nc == 0) return set_error(PG_INVALID_ARG, "coil combination: bad argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  DevBuf<float2> img;
  DevBuf<float> o;
  PG_TRY(img.upload((const float2*)coil_images, n * nc, s));
  PG_TRY(o.alloc(n));
  PG_LAUNCH(k_sum_magnitudes, ceil_div(n, 256), 256, 0, s, n, (int)nc, img.p, o.p);
  PG_CUDA(cudaMemcpyAsync(out, o.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

}  // extern "C"
