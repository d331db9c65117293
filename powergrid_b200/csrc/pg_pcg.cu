// PWLS-PCG on the device (solve_pwls_pcg.hpp:48-167) with the Robject
// regularizers (Robject.cpp:49-193, QuadPenalty.cpp:45-64, TVPenalty.cpp:43-68).
//
// Every vector op of an iteration is a kernel; inner products are
// accumulated in FP64: each block stores its partial sums and the block that
// finishes last adds all partials in a fixed order (so results are
// deterministic) and then evaluates the scalar step that follows (the CG
// coefficient, a Newton step, an early-exit test) in the same launch.  No
// step needs the host, so an iteration is replayed as one CUDA graph.
// Early exits set a device flag that turns the remaining kernels into
// no-ops, which returns the x of the exit point as the reference does.
//
// Segments: an operator may stack n_seg independent problems of equal size
// (the slices of a served request), x = [x_0; ...], y = [y_0; ...].  Every
// kernel then runs with blockIdx.y = segment over that segment's part of the
// vectors, with its own partial sums, last-block counter, FP64 scalars and
// flags, so each segment takes exactly the steps and early exits of its own
// solve (solve_pwls_pcg is run per slice by the reference's drivers,
// PowerGridIsmrmrd.cpp:191-264).  One segment is the plain solve.
//
// The regularizer is fused: Gradient = beta * sum_dims Ctd(dpot(Cd x)) is a
// 3-point stencil per dimension evaluated on the fly (no Cd/Ctd vectors),
// with the reference's boundary rules: Cd is zero below the offset and
// differences across row/slice boundaries (Robject.cpp:76-79); Ctd is
// d[j]-d[j+off] up to N-2-off, d[N-1-off] at N-1-off, zero above
// (Robject.cpp:111-117).
#include <cmath>
#include <cstring>
#include <vector>

#include <cooperative_groups.h>

#include "pg_ops.cuh"
#include "pg_profile.cuh"

namespace pg {

namespace {

struct PenDev {
  int kind;          // 0 quad, 1 TV
  int nd;            // dimensions penalised
  uint64_t N;
  uint64_t off[3];
  float beta, delta;
};

enum Scal { S_YWY = 0, S_OLD, S_GAMMA, S_DAWAD, S_DAWR, S_STEP, S_NEW, S_DIRDOT, S_PDEN, S_PDOT0, S_Q1, S_NSCAL };
enum Flag { F_DONE = 0, F_IT, F_COMPLETED, F_REASON, F_NFLAG };

constexpr int kRed = 256;  // threads per reduction block

__device__ __forceinline__ float2 dpot(const PenDev& R, float2 d) {
  if (R.kind == 0) return d;
  const float a = hypotf(d.x / R.delta, d.y / R.delta);
  const float s = sqrtf(1.f + a * a);
  return make_float2(d.x / s, d.y / s);
}
__device__ __forceinline__ float wpot(const PenDev& R, float2 d) {
  if (R.kind == 0) return 1.f;
  const float a = hypotf(d.x / R.delta, d.y / R.delta);
  return 1.f / sqrtf(1.f + a * a);
}

// Loads of the stencil helpers: plain, or through L2 only (CG) for data that
// other CTAs of the same launch wrote.
template <bool CG>
__device__ __forceinline__ float2 ldv(const float2* p, uint64_t i) {
  if constexpr (CG) return __ldcg(p + i);
  else return p[i];
}

template <bool CG = false>
__device__ __forceinline__ float2 zval(const float2* __restrict__ x, const float2* __restrict__ d, float st,
                                       uint64_t i) {
  const float2 a = ldv<CG>(x, i);
  if (!d) return a;
  const float2 b = ldv<CG>(d, i);
  return make_float2(a.x + st * b.x, a.y + st * b.y);
}

// beta * sum_dims Ctd(dpot(Cd z))[j], z = x + st*d.
template <bool CG = false>
__device__ __forceinline__ float2 grad_at(const PenDev& R, const float2* __restrict__ x, const float2* __restrict__ d,
                                          float st, uint64_t j) {
  float2 g = make_float2(0.f, 0.f);
  const float2 zj = zval<CG>(x, d, st, j);
  for (int dim = 0; dim < R.nd; ++dim) {
    const uint64_t off = R.off[dim];
    if (off >= R.N) continue;
    const uint64_t last = R.N - 1 - off;
    if (j > last) continue;
    float2 vj = make_float2(0.f, 0.f);
    if (j >= off) vj = dpot(R, csub(zj, zval<CG>(x, d, st, j - off)));
    if (j < last) {
      const float2 vn = dpot(R, csub(zval<CG>(x, d, st, j + off), zj));
      g = cadd(g, csub(vj, vn));
    } else {
      g = cadd(g, vj);
    }
  }
  return make_float2(R.beta * g.x, R.beta * g.y);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block reduction of NV values; thread 0 writes part[k*nb + blockIdx.x].
template <int NV>
__device__ __forceinline__ void block_store(const double (&v)[NV], double* part, int nb) {
  __shared__ double sv[NV][kRed / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    const double t = warp_sum(v[k]);
    if (l == 0) sv[k][w] = t;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = (l < (int)(blockDim.x >> 5)) ? sv[k][l] : 0.0;
      t = warp_sum(t);
      if (l == 0) part[(size_t)k * nb + blockIdx.x] = t;
    }
  }
}

// Block reduction of up to 2 values; thread 0 writes part[k*nb + blockIdx.x].
__device__ __forceinline__ void block_store2(double a, double b, double* part, int nb) {
  __shared__ double sa[kRed / 32], sb[kRed / 32];
  a = warp_sum(a);
  b = warp_sum(b);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sa[w] = a; sb[w] = b; }
  __syncthreads();
  if (w == 0) {
    a = (l < (int)(blockDim.x >> 5)) ? sa[l] : 0.0;
    b = (l < (int)(blockDim.x >> 5)) ? sb[l] : 0.0;
    a = warp_sum(a);
    b = warp_sum(b);
    if (l == 0) { part[blockIdx.x] = a; part[nb + blockIdx.x] = b; }
  }
}

// Fixed-order sum of part[k*nb .. k*nb+nb) by one warp.
__device__ __forceinline__ double part_sum(const double* part, int nb, int k) {
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += 32) v += part[k * nb + i];
  return warp_sum(v);
}

// ---- kernels ------------------------------------------------------------------
__global__ void k_fill_ones(uint64_t n, float* w) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w[i] = 1.f;
}

// sum W |y|^2 (norm_grad denominator, solve_pwls_pcg.hpp:42-46)
__global__ void k_ywy(uint64_t n, const float2* __restrict__ y, const float* __restrict__ W, double* part, int nb,
                      int pstride) {
  y += (uint64_t)blockIdx.y * n;
  W += (uint64_t)blockIdx.y * n;
  part += (size_t)blockIdx.y * pstride;
  double a = 0.0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float2 v = y[i];
    a += (double)W[i] * ((double)v.x * v.x + (double)v.y * v.y);
  }
  block_store2(a, 0.0, part, nb);
}

__global__ void k_scalar_init(const double* part, int nb, int pstride, double* sc, uint32_t* fl) {
  part += (size_t)blockIdx.x * pstride;
  sc += (size_t)blockIdx.x * S_NSCAL;
  fl += (size_t)blockIdx.x * F_NFLAG;
  const double ywy = part_sum(part, nb, 0);
  if (threadIdx.x == 0) {
    for (int i = 0; i < S_NSCAL; ++i) sc[i] = 0.0;
    sc[S_YWY] = ywy;
    fl[F_DONE] = 0; fl[F_IT] = 0; fl[F_COMPLETED] = 0; fl[F_REASON] = 0;
  }
}

// Last-block completion.  Every block has stored its partials (thread 0,
// inside block_store2); the block whose ticket is the last one then sees all
// of them.  The counter is reset for the next kernel of the stream.
__device__ __forceinline__ bool last_block(unsigned* counter) {
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
    if (last) *counter = 0u;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Fixed-order sum of part[k*nb .. k*nb+nb) by the whole (last) block.
__device__ __forceinline__ double block_part_sum(const double* part, int nb, int k) {
  __shared__ double red[kRed / 32];
  __shared__ double out;
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) v += __ldcg(part + (size_t)k * nb + i);
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    double r = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
    r = warp_sum(r);
    if (l == 0) out = r;
  }
  __syncthreads();
  const double res = out;
  __syncthreads();
  return res;
}

// r = W (.) (y - Ax): the residual before the first iteration.
__global__ void k_residual(uint64_t n, const float2* __restrict__ y, const float2* __restrict__ Ax,
                           const float* __restrict__ W, float2* __restrict__ r) {
  const uint64_t o = (uint64_t)blockIdx.y * n;
  y += o; Ax += o; W += o; r += o;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float2 d = csub(y[i], Ax[i]);
    const float w = W[i];
    r[i] = make_float2(w * d.x, w * d.y);
  }
}

// ngrad = A'r - R.Gradient(x); partials |A'r|^2 and |ngrad|^2; then the
// early exit on a vanishing gradient (:88-91) and the CG coefficient (:95-110).
// With ddir_prev set, the current direction is also copied there (the fused
// quadratic k_ddir reads neighbours of the old direction while it rewrites it).
__global__ void k_ngrad(PenDev R, const float2* __restrict__ x, float2* __restrict__ ngrad, double* part, int nb,
                        unsigned* counter, double* sc, uint32_t* fl, const float2* __restrict__ ddir,
                        float2* __restrict__ ddir_prev, int pstride) {
  pdl_wait();
  {
    const uint64_t o = (uint64_t)blockIdx.y * R.N;
    x += o; ngrad += o; ddir += o;
    if (ddir_prev) ddir_prev += o;
    part += (size_t)blockIdx.y * pstride; counter += blockIdx.y;
    sc += (size_t)blockIdx.y * S_NSCAL; fl += (size_t)blockIdx.y * F_NFLAG;
  }
  if (fl[F_DONE]) return;
  double a = 0.0, b = 0.0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < R.N; j += (uint64_t)gridDim.x * blockDim.x) {
    if (ddir_prev) ddir_prev[j] = ddir[j];
    const float2 raw = ngrad[j];
    a += (double)raw.x * raw.x + (double)raw.y * raw.y;
    const float2 g = grad_at(R, x, nullptr, 0.f, j);
    const float2 v = csub(raw, g);
    ngrad[j] = v;
    b += (double)v.x * v.x + (double)v.y * v.y;
  }
  block_store2(a, b, part, nb);
  if (!last_block(counter)) return;
  const double gn = block_part_sum(part, nb, 0);
  const double nw = block_part_sum(part, nb, 1);
  if (threadIdx.x == 0) {
    if (sqrt(gn) / sc[S_YWY] < 1e-10) { fl[F_DONE] = 1; fl[F_REASON] = 1; return; }
    double gamma = 0.0;
    if (fl[F_IT] > 0) gamma = (fabs(sc[S_OLD]) < 1e-10) ? 0.0 : nw / sc[S_OLD];
    sc[S_GAMMA] = gamma;
    sc[S_OLD] = nw;
  }
}

// ddir = ngrad + gamma ddir; partial Re<ddir, ngrad>; then the descent check (:113-116).
__global__ void k_ddir(uint64_t n, const float2* __restrict__ ngrad, float2* __restrict__ ddir, double* part, int nb,
                       unsigned* counter, double* sc, uint32_t* fl, int pstride) {
  pdl_wait();
  {
    const uint64_t o = (uint64_t)blockIdx.y * n;
    ngrad += o; ddir += o;
    part += (size_t)blockIdx.y * pstride; counter += blockIdx.y;
    sc += (size_t)blockIdx.y * S_NSCAL; fl += (size_t)blockIdx.y * F_NFLAG;
  }
  if (fl[F_DONE]) return;
  const float gm = (float)sc[S_GAMMA];
  double a = 0.0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const float2 g = ngrad[j];
    float2 d = ddir[j];
    d = make_float2(g.x + gm * d.x, g.y + gm * d.y);
    ddir[j] = d;
    a += (double)d.x * g.x + (double)d.y * g.y;
  }
  block_store2(a, 0.0, part, nb);
  if (!last_block(counter)) return;
  const double v = block_part_sum(part, nb, 0);
  if (threadIdx.x == 0) {
    sc[S_DIRDOT] = v;
    if (v < 0) { fl[F_DONE] = 1; fl[F_REASON] = 2; }
  }
}

// Quadratic penalty: ddir = ngrad + gamma ddir_prev, the descent product, and
// the sums the three Newton steps need (see newton_quad_steps) in one pass.
// Neighbour values of the new direction are formed from ngrad and ddir_prev,
// which this kernel does not write.
__global__ void k_ddir_quad(PenDev R, const float2* __restrict__ ngrad, const float2* __restrict__ ddir_prev,
                            float2* __restrict__ ddir, const float2* __restrict__ x, double* part, int nb,
                            unsigned* counter, double* sc, uint32_t* fl, int pstride) {
  pdl_wait();
  {
    const uint64_t o = (uint64_t)blockIdx.y * R.N;
    ngrad += o; ddir_prev += o; ddir += o; x += o;
    part += (size_t)blockIdx.y * pstride; counter += blockIdx.y;
    sc += (size_t)blockIdx.y * S_NSCAL; fl += (size_t)blockIdx.y * F_NFLAG;
  }
  if (fl[F_DONE]) return;
  const float gm = (float)sc[S_GAMMA];
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < R.N; j += (uint64_t)gridDim.x * blockDim.x) {
    const float2 g = ngrad[j];
    const float2 dj = zval(ngrad, ddir_prev, gm, j);
    ddir[j] = dj;
    v[0] += (double)dj.x * g.x + (double)dj.y * g.y;
    for (int dim = 0; dim < R.nd; ++dim) {
      const uint64_t off = R.off[dim];
      if (j < off || off >= R.N) continue;
      const float2 cd = csub(dj, zval(ngrad, ddir_prev, gm, j - off));
      v[1] += (double)cd.x * cd.x + (double)cd.y * cd.y;
    }
    const float2 gx = grad_at(R, x, nullptr, 0.f, j);
    const float2 gd = grad_at(R, ngrad, ddir_prev, gm, j);
    v[2] += (double)dj.x * gx.x + (double)dj.y * gx.y;
    v[3] += (double)dj.x * gd.x + (double)dj.y * gd.y;
  }
  block_store<4>(v, part, nb);
  if (!last_block(counter)) return;
  const double dot = block_part_sum(part, nb, 0);
  const double pden = block_part_sum(part, nb, 1);
  const double pdot0 = block_part_sum(part, nb, 2);
  const double q1 = block_part_sum(part, nb, 3);
  if (threadIdx.x == 0) {
    sc[S_DIRDOT] = dot;
    sc[S_PDEN] = pden;
    sc[S_PDOT0] = pdot0;
    sc[S_Q1] = q1;
    if (dot < 0) { fl[F_DONE] = 1; fl[F_REASON] = 2; }
  }
}

// k_ngrad followed by k_ddir_quad in one launch, for images of at most
// kImgMax voxels: one cluster of kImgCL CTAs covers a whole image (one cluster
// per segment of a stacked solve), so the grid-wide step between the two (the CG coefficient needs the
// sum over all voxels) is a cluster barrier instead of a kernel boundary and a
// last-block reduction.  It pays while the image fits one voxel per thread:
// at 64x64 a solve ran 4.4 % faster (19.7k vs 18.9k iterations/s, measured
// with 1024-thread CTAs), while at 128x128 the two kernels over 64 SMs won
// (8.77k vs 8.55k with two voxels per thread, 8.61k with a 16-CTA cluster).  Each CTA sums the CTAs' partials itself, in rank
// order, so every CTA holds the same FP64 totals and the same coefficient.
// Same per-voxel arithmetic as the two kernels; the FP64 sums are added in a
// different (fixed) order.
namespace cgx = cooperative_groups;
// 512-thread CTAs (32K registers, half an SM) so that a cluster never needs
// whole idle SMs while other streams' kernels run.
constexpr int kImgCL = 8, kImgT = 512, kImgPer = 1;
constexpr uint64_t kImgMax = (uint64_t)kImgCL * kImgT * kImgPer;

// Sum of NV doubles over the CTA into red[0..NV) (thread 0 writes; all threads
// must call it; ends with a barrier).
template <int NV>
__device__ __forceinline__ void cta_sum(double (&v)[NV], double* red) {
  __shared__ double sw[NV][kImgT / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    const double t = warp_sum(v[k]);
    if (l == 0) sw[k][w] = t;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = (l < kImgT / 32) ? sw[k][l] : 0.0;
      t = warp_sum(t);
      if (l == 0) red[k] = t;
    }
  }
  __syncthreads();
}

// Totals over the cluster's CTAs, added in rank order (identical in every CTA).
template <int NV>
__device__ __forceinline__ void cluster_totals(cgx::cluster_group& cl, double* red, double (&tot)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; ++k) tot[k] = 0.0;
  for (int q = 0; q < kImgCL; ++q) {
    const double* rq = cl.map_shared_rank(red, q);
#pragma unroll
    for (int k = 0; k < NV; ++k) tot[k] += rq[k];
  }
}

__global__ void __launch_bounds__(kImgT, 2)
    k_image_step_quad(PenDev R, const float2* __restrict__ x, float2* ngrad, float2* ddir, float2* ddir_prev,
                      double* sc, uint32_t* fl) {
  pdl_wait();
  {  // cluster blockIdx.y solves segment blockIdx.y: its part of the vectors, its scalars and flags
    const uint64_t o = (uint64_t)blockIdx.y * R.N;
    x += o; ngrad += o; ddir += o; ddir_prev += o;
    sc += (size_t)blockIdx.y * S_NSCAL; fl += (size_t)blockIdx.y * F_NFLAG;
  }
  cgx::cluster_group cl = cgx::this_cluster();
  __shared__ double redA[2], redB[4];
  const bool done0 = fl[F_DONE] != 0;     // the same value in every CTA
  const uint64_t stride = (uint64_t)kImgCL * kImgT;
  const uint64_t t0 = (uint64_t)cl.block_rank() * kImgT + threadIdx.x;
  if (!done0) {
    // gradient: ngrad = A'r - R.Gradient(x), the previous direction kept (k_ngrad)
    double v[2] = {0.0, 0.0};
    for (uint64_t j = t0; j < R.N; j += stride) {
      ddir_prev[j] = ddir[j];
      const float2 raw = ngrad[j];
      v[0] += (double)raw.x * raw.x + (double)raw.y * raw.y;
      const float2 g = grad_at(R, x, nullptr, 0.f, j);
      const float2 u = csub(raw, g);
      ngrad[j] = u;
      v[1] += (double)u.x * u.x + (double)u.y * u.y;
    }
    cta_sum<2>(v, redA);
  }
  cl.sync();   // every CTA's ngrad / ddir_prev writes and partials are visible cluster-wide
  bool done = done0;
  float gm = 0.f;
  if (!done) {
    double tot[2];
    cluster_totals<2>(cl, redA, tot);
    const double gn = tot[0], nw = tot[1];
    if (sqrt(gn) / sc[S_YWY] < 1e-10) {
      done = true;
      if (cl.block_rank() == 0 && threadIdx.x == 0) { fl[F_DONE] = 1; fl[F_REASON] = 1; }
    } else {
      double gamma = 0.0;
      if (fl[F_IT] > 0) gamma = (fabs(sc[S_OLD]) < 1e-10) ? 0.0 : nw / sc[S_OLD];
      gm = (float)gamma;
      cl.sync();   // every CTA has read sc[S_OLD] before rank 0 replaces it
      if (cl.block_rank() == 0 && threadIdx.x == 0) { sc[S_GAMMA] = gamma; sc[S_OLD] = nw; }
    }
  }
  if (!done) {
    // direction and the quadratic line-search sums (k_ddir_quad)
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    // ngrad and ddir_prev at neighbouring voxels come from other CTAs: L2 loads
    for (uint64_t j = t0; j < R.N; j += stride) {
      const float2 g = ldv<true>(ngrad, j);
      const float2 dj = zval<true>(ngrad, ddir_prev, gm, j);
      ddir[j] = dj;
      v[0] += (double)dj.x * g.x + (double)dj.y * g.y;
      for (int dim = 0; dim < R.nd; ++dim) {
        const uint64_t off = R.off[dim];
        if (j < off || off >= R.N) continue;
        const float2 cd = csub(dj, zval<true>(ngrad, ddir_prev, gm, j - off));
        v[1] += (double)cd.x * cd.x + (double)cd.y * cd.y;
      }
      const float2 gx = grad_at(R, x, nullptr, 0.f, j);
      const float2 gd = grad_at<true>(R, ngrad, ddir_prev, gm, j);
      v[2] += (double)dj.x * gx.x + (double)dj.y * gx.y;
      v[3] += (double)dj.x * gd.x + (double)dj.y * gd.y;
    }
    cta_sum<4>(v, redB);
    cl.sync();
    double tot[4];
    cluster_totals<4>(cl, redB, tot);
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
      sc[S_DIRDOT] = tot[0];
      sc[S_PDEN] = tot[1];
      sc[S_PDOT0] = tot[2];
      sc[S_Q1] = tot[3];
      if (tot[0] < 0) { fl[F_DONE] = 1; fl[F_REASON] = 2; }
    }
  }
  cl.sync();   // no CTA leaves while another reads its shared memory
}

// k_daw followed by k_update in one launch, for data and images of at most
// kImgMax entries per segment (quadratic penalty; one cluster per segment): the line-search sums,
// the three Newton steps (newton_quad_steps, evaluated by every CTA from the
// same rank-ordered totals) and the update of x, Ax and the residual, with a
// cluster barrier where the two kernels had a launch boundary.
__global__ void __launch_bounds__(kImgT, 2)
    k_data_step_quad(uint64_t ni, uint64_t nd, float2* x, const float2* __restrict__ ddir, float2* Ax,
                     const float2* __restrict__ Adir, const float2* __restrict__ y, const float* __restrict__ W,
                     float2* r, double beta, double* sc, uint32_t* fl) {
  pdl_wait();
  {  // cluster blockIdx.y solves segment blockIdx.y
    const uint64_t oi = (uint64_t)blockIdx.y * ni, od = (uint64_t)blockIdx.y * nd;
    x += oi; ddir += oi;
    Ax += od; Adir += od; y += od; W += od; r += od;
    sc += (size_t)blockIdx.y * S_NSCAL; fl += (size_t)blockIdx.y * F_NFLAG;
  }
  cgx::cluster_group cl = cgx::this_cluster();
  __shared__ double red[2];
  const bool done0 = fl[F_DONE] != 0;     // the same value in every CTA
  const uint64_t stride = (uint64_t)kImgCL * kImgT;
  const uint64_t t0 = (uint64_t)cl.block_rank() * kImgT + threadIdx.x;
  if (!done0) {
    // dAWAd = Re<Adir, W Adir>, dAWr = Re(Adir' r) (k_daw)
    double v[2] = {0.0, 0.0};
    for (uint64_t i = t0; i < nd; i += stride) {
      const float2 a = Adir[i];
      const float2 q = r[i];
      v[0] += (double)W[i] * ((double)a.x * a.x + (double)a.y * a.y);
      v[1] += (double)a.x * q.x + (double)a.y * q.y;
    }
    cta_sum<2>(v, red);
  }
  cl.sync();
  bool done = done0;
  float st = 0.f;
  if (!done) {
    double tot[2];
    cluster_totals<2>(cl, red, tot);
    const double dawad = tot[0], dawr = tot[1];
    const double denom = dawad + beta * sc[S_PDEN];
    double step = 0.0;
    bool bad = false;
    for (int k = 0; k < 3; ++k) {                 // newton_quad_steps
      if (fabs(denom) < 1e-20 || fabs(denom) > 1e25 || denom != denom) { bad = true; break; }
      const double pdot = sc[S_PDOT0] + step * sc[S_Q1];
      step = step - (-dawr + step * dawad + pdot) / denom;
    }
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
      sc[S_DAWAD] = dawad;
      sc[S_DAWR] = dawr;
      sc[S_STEP] = step;
      if (bad) { fl[F_DONE] = 1; fl[F_REASON] = 3; }
    }
    done = bad;
    st = (float)step;
  }
  if (!done) {
    // x += step ddir; Ax += step Adir; r = W (.) (y - Ax) (k_update)
    const uint64_t n = ni > nd ? ni : nd;
    for (uint64_t i = t0; i < n; i += stride) {
      if (i < ni) { const float2 d = ddir[i]; float2 v = x[i]; v.x += st * d.x; v.y += st * d.y; x[i] = v; }
      if (i < nd) {
        const float2 d = Adir[i];
        float2 v = Ax[i];
        v.x += st * d.x; v.y += st * d.y;
        Ax[i] = v;
        const float2 e = csub(y[i], v);
        const float w = W[i];
        r[i] = make_float2(w * e.x, w * e.y);
      }
    }
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
      fl[F_IT] += 1;
      fl[F_COMPLETED] = fl[F_IT];
    }
  }
  cl.sync();   // no CTA leaves while another reads its shared memory
}

// The three Newton steps of the quadratic penalty (:132-150) from the sums
// k_ddir_quad stored: Gradient is linear and wpot = 1, so pdenom is fixed and
// pdot(s) = pdot(0) + s Re<ddir, Gradient(ddir)>.
__device__ __forceinline__ void newton_quad_steps(double beta, double* sc, uint32_t* fl) {
  const double denom = sc[S_DAWAD] + beta * sc[S_PDEN];
  double step = 0.0;
  for (int k = 0; k < 3; ++k) {
    if (fabs(denom) < 1e-20 || fabs(denom) > 1e25 || denom != denom) {
      sc[S_STEP] = step;
      fl[F_DONE] = 1;
      fl[F_REASON] = 3;
      return;
    }
    const double pdot = sc[S_PDOT0] + step * sc[S_Q1];
    step = step - (-sc[S_DAWR] + step * sc[S_DAWAD] + pdot) / denom;
  }
  sc[S_STEP] = step;
}

// dAWAd = Re<Adir, W Adir>, dAWr = Re(Adir' r) (:123-125).
__global__ void k_daw(uint64_t n, const float2* __restrict__ Adir, const float* __restrict__ W,
                      const float2* __restrict__ r, double* part, int nb, unsigned* counter, double* sc,
                      uint32_t* fl, int quad, double beta, int pstride) {
  pdl_wait();
  {
    const uint64_t o = (uint64_t)blockIdx.y * n;
    Adir += o; W += o; r += o;
    part += (size_t)blockIdx.y * pstride; counter += blockIdx.y;
    sc += (size_t)blockIdx.y * S_NSCAL; fl += (size_t)blockIdx.y * F_NFLAG;
  }
  if (fl[F_DONE]) return;
  double a = 0.0, b = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // four elements per round with every load issued first (latency-bound at these sizes)
  for (; i + 3 * stride < n; i += 4 * stride) {
    float2 v[4], q[4];
    float w[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) { v[u] = Adir[i + u * stride]; q[u] = r[i + u * stride]; w[u] = W[i + u * stride]; }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a += (double)w[u] * ((double)v[u].x * v[u].x + (double)v[u].y * v[u].y);
      b += (double)v[u].x * q[u].x + (double)v[u].y * q[u].y;
    }
  }
  for (; i < n; i += stride) {
    const float2 v = Adir[i];
    const float2 q = r[i];
    a += (double)W[i] * ((double)v.x * v.x + (double)v.y * v.y);
    b += (double)v.x * q.x + (double)v.y * q.y;
  }
  block_store2(a, b, part, nb);
  if (!last_block(counter)) return;
  const double sa = block_part_sum(part, nb, 0);
  const double sb = block_part_sum(part, nb, 1);
  if (threadIdx.x == 0) {
    sc[S_DAWAD] = sa;
    sc[S_DAWR] = sb;
    sc[S_STEP] = 0.0;
    if (quad) newton_quad_steps(beta, sc, fl);
  }
}

// One Newton step at z = x + step*ddir (:132-150): pdenom = sum_dims sum
// wpot(Cd z) |Cd ddir|^2, pdot = Re<ddir, Gradient(z)>, then the step update.
__global__ void k_newton(PenDev R, const float2* __restrict__ x, const float2* __restrict__ ddir, double beta,
                         double* part, int nb, unsigned* counter, double* sc, uint32_t* fl, int pstride) {
  pdl_wait();
  {
    const uint64_t o = (uint64_t)blockIdx.y * R.N;
    x += o; ddir += o;
    part += (size_t)blockIdx.y * pstride; counter += blockIdx.y;
    sc += (size_t)blockIdx.y * S_NSCAL; fl += (size_t)blockIdx.y * F_NFLAG;
  }
  if (fl[F_DONE]) return;
  const float st = (float)sc[S_STEP];
  double a = 0.0, b = 0.0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < R.N; j += (uint64_t)gridDim.x * blockDim.x) {
    const float2 dj = ddir[j];
    const float2 zj = zval(x, ddir, st, j);
    for (int dim = 0; dim < R.nd; ++dim) {
      const uint64_t off = R.off[dim];
      if (j < off || off >= R.N) continue;
      const float2 cd = csub(dj, ddir[j - off]);
      const float2 cz = csub(zj, zval(x, ddir, st, j - off));
      a += (double)wpot(R, cz) * ((double)cd.x * cd.x + (double)cd.y * cd.y);
    }
    const float2 g = grad_at(R, x, ddir, st, j);
    b += (double)dj.x * g.x + (double)dj.y * g.y;
  }
  block_store2(a, b, part, nb);
  if (!last_block(counter)) return;
  const double pden = block_part_sum(part, nb, 0);
  const double pdot = block_part_sum(part, nb, 1);
  if (threadIdx.x == 0) {
    const double denom = sc[S_DAWAD] + beta * pden;
    if (fabs(denom) < 1e-20 || fabs(denom) > 1e25 || denom != denom) { fl[F_DONE] = 1; fl[F_REASON] = 3; return; }
    const double step = sc[S_STEP];
    sc[S_STEP] = step - (-sc[S_DAWR] + step * sc[S_DAWAD] + pdot) / denom;
  }
}

// x += step ddir; Ax += step Adir (:160-161); the next residual
// r = W (.) (y - Ax) in the same pass; then the iteration count.
__global__ void k_update(uint64_t ni, uint64_t nd, float2* __restrict__ x, const float2* __restrict__ ddir,
                         float2* __restrict__ Ax, const float2* __restrict__ Adir, const float2* __restrict__ y,
                         const float* __restrict__ W, float2* __restrict__ r, const double* sc, uint32_t* fl) {
  pdl_wait();
  {
    const uint64_t oi = (uint64_t)blockIdx.y * ni, od = (uint64_t)blockIdx.y * nd;
    x += oi; ddir += oi;
    Ax += od; Adir += od; y += od; W += od; r += od;
    sc += (size_t)blockIdx.y * S_NSCAL; fl += (size_t)blockIdx.y * F_NFLAG;
  }
  if (fl[F_DONE]) return;
  const float st = (float)sc[S_STEP];
  const uint64_t n = ni > nd ? ni : nd;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (i < ni) { const float2 d = ddir[i]; float2 v = x[i]; v.x += st * d.x; v.y += st * d.y; x[i] = v; }
    if (i < nd) {
      const float2 d = Adir[i];
      float2 v = Ax[i];
      v.x += st * d.x; v.y += st * d.y;
      Ax[i] = v;
      const float2 e = csub(y[i], v);
      const float w = W[i];
      r[i] = make_float2(w * e.x, w * e.y);
    }
  }
  // the count needs no other block's data: block 0 takes it
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    fl[F_IT] += 1;
    fl[F_COMPLETED] = fl[F_IT];
  }
}

// Completed iterations of each segment (out: nseg values).
__global__ void k_copy_iters(const uint32_t* fl, int nseg, uint32_t* out) {
  for (int g = threadIdx.x; g < nseg; g += blockDim.x) out[g] = fl[(size_t)g * F_NFLAG + F_COMPLETED];
}

// One element per thread up to 4 blocks per SM, then grid-stride: small
// vectors still spread over many SMs, large ones keep the partial count low.
int red_blocks(uint64_t n) {
  uint64_t b = (n + kRed - 1) / kRed;
  if (b > 592) b = 592;
  if (b < 1) b = 1;
  return (int)b;
}

PenDev make_pen(const pg_penalty& R) {
  PenDev p{};
  p.kind = R.kind;
  p.N = R.nx * R.ny * R.nz;
  p.nd = (R.nz == 1 || R.dims2penalize == 2) ? 2 : 3;  // Robject.cpp:128-132
  p.off[0] = 1;
  p.off[1] = R.ny;
  p.off[2] = R.nx * R.ny;
  p.beta = R.beta;
  p.delta = R.delta;
  return p;
}

// Whether k_image_step_quad can run: one cluster of kImgCL CTAs of kImgT
// threads must fit (checked once); PG_IMAGE_STEP=0 keeps the two kernels.
bool image_step_ok() {
  static const bool ok = [] {
    const char* e = getenv("PG_IMAGE_STEP");
    if (e && e[0] == '0') return false;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kImgCL, 1, 1);
    cfg.blockDim = dim3(kImgT, 1, 1);
    cudaLaunchAttribute a[1];
    a[0].id = cudaLaunchAttributeClusterDimension;
    a[0].val.clusterDim.x = kImgCL;
    a[0].val.clusterDim.y = 1;
    a[0].val.clusterDim.z = 1;
    cfg.attrs = a;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_image_step_quad, &cfg) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return n >= 1;
  }();
  return ok;
}

pg_status launch_data_step(int nseg, uint64_t ni, uint64_t nd, float2* x, const float2* ddir, float2* Ax,
                           const float2* Adir, const float2* y, const float* W, float2* r, double beta, double* sc,
                           uint32_t* fl, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kImgCL, (unsigned)nseg, 1);   // one cluster per segment
  cfg.blockDim = dim3(kImgT, 1, 1);
  cfg.stream = s;
  cudaLaunchAttribute a[2];
  a[0].id = cudaLaunchAttributeClusterDimension;
  a[0].val.clusterDim.x = kImgCL;
  a[0].val.clusterDim.y = 1;
  a[0].val.clusterDim.z = 1;
  a[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;   // the kernel calls pdl_wait()
  a[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = a;
  cfg.numAttrs = 2;
  PG_CUDA(cudaLaunchKernelEx(&cfg, k_data_step_quad, ni, nd, x, ddir, Ax, Adir, y, W, r, beta, sc, fl));
  count_launch();
  return PG_OK;
}

pg_status launch_image_step(int nseg, const PenDev& R, const float2* x, float2* ngrad, float2* ddir,
                            float2* ddir_prev, double* sc, uint32_t* fl, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kImgCL, (unsigned)nseg, 1);   // one cluster per segment
  cfg.blockDim = dim3(kImgT, 1, 1);
  cfg.stream = s;
  cudaLaunchAttribute a[2];
  a[0].id = cudaLaunchAttributeClusterDimension;
  a[0].val.clusterDim.x = kImgCL;
  a[0].val.clusterDim.y = 1;
  a[0].val.clusterDim.z = 1;
  a[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;   // the kernel calls pdl_wait()
  a[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = a;
  cfg.numAttrs = 2;
  PG_CUDA(cudaLaunchKernelEx(&cfg, k_image_step_quad, R, x, ngrad, ddir, ddir_prev, sc, fl));
  count_launch();
  return PG_OK;
}

struct Solver {
  pg_op A;
  uint64_t nd, ni;      // per-segment data and image lengths
  int nseg = 1;         // independent problems stacked in the vectors
  int pstride = 0;      // doubles of partial sums per segment
  PenDev R;
  double beta;
  DevBuf<float2> x, Ax, r, ngrad, ddir, Adir, ddir_prev;
  DevBuf<float> Wones;
  DevBuf<double> part, sc;
  DevBuf<uint32_t> fl;
  DevBuf<unsigned> counter;   // last-block ticket, zero between kernels
  const float2* y;
  const float* W;
  int nbd, nbi;

  // One PCG iteration; r = W (.) (y - Ax) holds on entry and on exit.
  pg_status iteration(cudaStream_t s) {
    const dim3 gd((unsigned)nbd, (unsigned)nseg), gi((unsigned)nbi, (unsigned)nseg);
    const bool quad = R.kind == 0;
    PG_TRY(A->adjoint(r.p, ngrad.p, s));
    if (quad && R.N <= kImgMax && image_step_ok()) {
      // gradient and direction of small images in one launch, one cluster per segment
      PG_TRY(launch_image_step(nseg, R, x.p, ngrad.p, ddir.p, ddir_prev.p, sc.p, fl.p, s));
    } else {
      PG_LAUNCH_PDL(k_ngrad, gi, kRed, 0, s, R, x.p, ngrad.p, part.p, nbi, counter.p, sc.p, fl.p, ddir.p,
                    quad ? ddir_prev.p : nullptr, pstride);
      if (quad)
        PG_LAUNCH_PDL(k_ddir_quad, gi, kRed, 0, s, R, ngrad.p, ddir_prev.p, ddir.p, x.p, part.p, nbi, counter.p,
                      sc.p, fl.p, pstride);
      else
        PG_LAUNCH_PDL(k_ddir, gi, kRed, 0, s, ni, ngrad.p, ddir.p, part.p, nbi, counter.p, sc.p, fl.p, pstride);
    }
    PG_TRY(A->forward(ddir.p, Adir.p, s));
    if (quad && nd <= kImgMax && ni <= kImgMax && image_step_ok()) {
      // line search and update of small problems in one launch, one cluster per segment
      return launch_data_step(nseg, ni, nd, x.p, ddir.p, Ax.p, Adir.p, y, W, r.p, beta, sc.p, fl.p, s);
    }
    PG_LAUNCH_PDL(k_daw, gd, kRed, 0, s, nd, Adir.p, W, r.p, part.p, nbd, counter.p, sc.p, fl.p, quad ? 1 : 0, beta,
              pstride);
    if (!quad)
      for (int k = 0; k < 3; ++k)
        PG_LAUNCH_PDL(k_newton, gi, kRed, 0, s, R, x.p, ddir.p, beta, part.p, nbi, counter.p, sc.p, fl.p, pstride);
    PG_LAUNCH_PDL(k_update, dim3((unsigned)red_blocks(std::max(nd, ni)), (unsigned)nseg), kRed, 0, s, ni, nd, x.p,
              ddir.p, Ax.p, Adir.p, y, W, r.p, sc.p, fl.p);
    return PG_OK;
  }
};

constexpr int kChunk = 4;   // PCG iterations per chunk graph

bool graphs_enabled() {
  const char* e = getenv("PG_NO_GRAPH");
  return !(e && e[0] == '1');
}

}  // namespace

namespace {

// Solver buffers and the instantiated per-iteration graph, cached on the
// operator.  The graph reads y and W from ybuf / wbuf, so a new solve only
// copies its inputs there and replays the graph.
struct PcgCache : pg_pcg_cache_base {
  Solver S;
  DevBuf<float2> ybuf;
  DevBuf<float> wbuf;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // With stage timing on, `exec` is captured without stage events and
  // `exec_timed` with them; a solve replays the timed copy for its last
  // iteration only (event nodes in every iteration cost ~10 us each).
  cudaGraph_t graph_timed = nullptr;
  cudaGraphExec_t exec_timed = nullptr;
  // kChunk iterations in one graph: one launch gap per chunk instead of per
  // iteration (0.7 % of a cfg2 solve).  Captured on the cache's second
  // solve: a one-off solve (a served job) would pay the capture and the
  // instantiation, ~ms, for microseconds.
  cudaGraph_t graph_chunk = nullptr;
  cudaGraphExec_t exec_chunk = nullptr;
  uint64_t per_iter = 0;
  uint64_t solves = 0;
  pg_penalty R{};
  uint64_t prof_epoch = 0;
  bool w_ones = true;
  ~PcgCache() override {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (exec_timed) cudaGraphExecDestroy(exec_timed);
    if (graph_timed) cudaGraphDestroy(graph_timed);
    if (exec_chunk) cudaGraphExecDestroy(exec_chunk);
    if (graph_chunk) cudaGraphDestroy(graph_chunk);
  }
  bool same_penalty(const pg_penalty& r) const {
    return R.kind == r.kind && R.nx == r.nx && R.ny == r.ny && R.nz == r.nz && R.beta == r.beta &&
           R.delta == r.delta && R.dims2penalize == r.dims2penalize;
  }
  bool matches(const pg_penalty& r, bool ones) const {
    return R.kind == r.kind && R.nx == r.nx && R.ny == r.ny && R.nz == r.nz && R.beta == r.beta &&
           R.delta == r.delta && R.dims2penalize == r.dims2penalize && prof_epoch == g_profile_epoch &&
           w_ones == ones;
  }
};

pg_status make_cache(pg_op_s* A, const pg_penalty& Rh, bool w_ones, std::unique_ptr<PcgCache>* out, cudaStream_t s) {
  auto c = std::make_unique<PcgCache>();
  Solver& S = c->S;
  const uint64_t g = A->n_seg ? A->n_seg : 1;
  S.A = A;
  S.nseg = (int)g;
  S.nd = A->n_data / g;
  S.ni = A->n_image / g;
  S.R = make_pen(Rh);
  S.beta = Rh.beta;
  S.nbd = red_blocks(S.nd);
  S.nbi = red_blocks(S.ni);
  const int nb = std::max(S.nbd, S.nbi);
  S.pstride = 4 * nb;
  PG_TRY(S.x.alloc(A->n_image));
  PG_TRY(S.Ax.alloc(A->n_data));
  PG_TRY(S.r.alloc(A->n_data));
  PG_TRY(S.ngrad.alloc(A->n_image));
  PG_TRY(S.ddir.alloc(A->n_image));
  if (Rh.kind == PG_PENALTY_QUAD) PG_TRY(S.ddir_prev.alloc(A->n_image));
  PG_TRY(S.Adir.alloc(A->n_data));
  PG_TRY(S.part.alloc((uint64_t)S.pstride * g));
  PG_TRY(S.sc.alloc(S_NSCAL * g));
  PG_TRY(S.fl.alloc(F_NFLAG * g));
  PG_TRY(S.counter.alloc(g));
  PG_CUDA(cudaMemsetAsync(S.counter.p, 0, g * sizeof(unsigned), s));
  PG_TRY(c->ybuf.alloc(A->n_data));
  PG_TRY(c->wbuf.alloc(A->n_data));
  if (w_ones) PG_LAUNCH(k_fill_ones, ceil_div(A->n_data, 256), 256, 0, s, A->n_data, c->wbuf.p);
  S.y = c->ybuf.p;
  S.W = c->wbuf.p;
  c->R = Rh;
  c->prof_epoch = g_profile_epoch;
  c->w_ones = w_ones;
  *out = std::move(c);
  return PG_OK;
}

}  // namespace

pg_status pcg_iterate(pg_op_s* A, PcgCache* cache, uint64_t niter, float2* xout, uint32_t* iters_dev,
                      cudaStream_t s, const std::atomic<bool>* cancel);

pg_status pcg_solve_device(pg_op_s* A, const float2* x0, const float* W, const float2* y, const pg_penalty& Rh,
                           uint64_t niter, float2* xout, uint32_t* iters_dev, cudaStream_t s,
                           const std::atomic<bool>* cancel, bool resume) {
  const uint64_t ni = A->n_image, nd = A->n_data;
  const uint64_t nseg = A->n_seg ? A->n_seg : 1;
  if (Rh.nx * Rh.ny * Rh.nz * nseg != ni)
    return set_error(PG_INVALID_ARG, "penalty size %llux%llux%llu does not match the image length %llu",
                     (unsigned long long)Rh.nx, (unsigned long long)Rh.ny, (unsigned long long)Rh.nz,
                     (unsigned long long)(ni / nseg));
  if (Rh.kind != PG_PENALTY_QUAD && Rh.kind != PG_PENALTY_TV) return set_error(PG_INVALID_ARG, "unknown penalty");
  if (Rh.kind == PG_PENALTY_TV && !(Rh.delta > 0)) return set_error(PG_INVALID_ARG, "TV penalty needs delta > 0");

  auto* cache = dynamic_cast<PcgCache*>(A->pcg_cache.get());
  if (resume) {
    // continue from the state on the operator (a solve or pg_pcg_state_load)
    if (!cache || !cache->same_penalty(Rh))
      return set_error(PG_INVALID_ARG, "pcg resume: no solver state for this penalty on the operator");
    PG_CUDA(cudaMemcpyAsync(cache->ybuf.p, y, nd * sizeof(float2), cudaMemcpyDeviceToDevice, s));
    if (W) PG_CUDA(cudaMemcpyAsync(cache->wbuf.p, W, nd * sizeof(float), cudaMemcpyDeviceToDevice, s));
    else PG_LAUNCH(k_fill_ones, ceil_div(nd, 256), 256, 0, s, nd, cache->wbuf.p);
    // what wbuf holds now: a later plain solve reuses the cache only if it is ones
    cache->w_ones = (W == nullptr);
    return pcg_iterate(A, cache, niter, xout, iters_dev, s, cancel);
  }
  if (!cache || !cache->matches(Rh, W == nullptr)) {
    A->pcg_cache.reset();
    std::unique_ptr<PcgCache> c;
    PG_TRY(make_cache(A, Rh, W == nullptr, &c, s));
    cache = c.get();
    A->pcg_cache = std::move(c);
  }
  Solver& S = cache->S;
  // inputs into the buffers the graph reads
  PG_CUDA(cudaMemcpyAsync(cache->ybuf.p, y, nd * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  if (W) PG_CUDA(cudaMemcpyAsync(cache->wbuf.p, W, nd * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if (x0) PG_CUDA(cudaMemcpyAsync(S.x.p, x0, ni * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  else PG_CUDA(cudaMemsetAsync(S.x.p, 0, ni * sizeof(float2), s));
  PG_CUDA(cudaMemsetAsync(S.ddir.p, 0, ni * sizeof(float2), s));
  // Ax = A * xInitial (:55).  Without x0 the start is zero and so is A * 0,
  // exactly (the operators are linear and their factors finite: the
  // deapodization's NaNs are stored as 0), so Ax is cleared instead.
  pg_status st = PG_OK;
  if (x0) st = A->forward(S.x.p, S.Ax.p, s);
  else PG_CUDA(cudaMemsetAsync(S.Ax.p, 0, nd * sizeof(float2), s));
  if (st != PG_OK) { A->pcg_cache.reset(); return st; }
  PG_LAUNCH(k_ywy, dim3((unsigned)S.nbd, (unsigned)S.nseg), kRed, 0, s, S.nd, S.y, S.W, S.part.p, S.nbd, S.pstride);
  PG_LAUNCH(k_scalar_init, (unsigned)S.nseg, 32, 0, s, S.part.p, S.nbd, S.pstride, S.sc.p, S.fl.p);
  PG_LAUNCH(k_residual, dim3((unsigned)S.nbd, (unsigned)S.nseg), kRed, 0, s, S.nd, S.y, S.Ax.p, S.W, S.r.p);
  return pcg_iterate(A, cache, niter, xout, iters_dev, s, cancel);
}

// kChunk iterations captured as one graph, after the one-iteration graph
// exists; on any failure the solve goes on with the one-iteration graph.
void capture_chunk(PcgCache* cache, cudaStream_t s) {
  const uint64_t before = g_launches.load();
  g_profile_suppress = true;
  pg_status st = PG_OK;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    for (int k = 0; k < kChunk && st == PG_OK; ++k) st = cache->S.iteration(s);
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (st == PG_OK && ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
    if (st == PG_OK && ce == cudaSuccess) {
      cache->graph_chunk = graph;
      cache->exec_chunk = exec;
      graph = nullptr;
    }
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
  g_profile_suppress = false;
  // the capture counted launches that never ran
  g_launches.fetch_sub(g_launches.load() - before);
}

// The iterations of a solve, from the state in the cache.
pg_status pcg_iterate(pg_op_s* A, PcgCache* cache, uint64_t niter, float2* xout, uint32_t* iters_dev,
                      cudaStream_t s, const std::atomic<bool>* cancel) {
  Solver& S = cache->S;
  const uint64_t ni = A->n_image;
  pg_status st = PG_OK;
  uint64_t it = 0;
  if (!cache->exec && niter > 0) {
    // first iteration eagerly: allocates every workspace the graph will use
    st = S.iteration(s);
    if (st != PG_OK) { A->pcg_cache.reset(); return st; }
    it = 1;
    if (graphs_enabled() && niter > 1) {
      // one capture without stage events, and with stage timing on a second
      // one with them
      for (int timed = 0; timed < (g_profile ? 2 : 1); ++timed) {
        const uint64_t before = g_launches.load();
        g_profile_suppress = timed == 0;
        PG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        st = S.iteration(s);
        cudaGraph_t graph = nullptr;
        cudaError_t ce = cudaStreamEndCapture(s, &graph);
        g_profile_suppress = false;
        // the capture pass counted launches that never ran
        cache->per_iter = g_launches.load() - before;
        g_launches.fetch_sub(cache->per_iter);
        if (st != PG_OK) {
          if (graph) cudaGraphDestroy(graph);
          cudaGetLastError();
          A->pcg_cache.reset();
          return st;
        }
        cudaGraphExec_t exec = nullptr;
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
        if (ce != cudaSuccess) {
          // The capture or its instantiation failed; the captured work never
          // ran, so the state is the one after the eager iteration: go on
          // without graphs (same kernels, launched one by one).
          if (graph) cudaGraphDestroy(graph);
          cudaGetLastError();
          if (cache->exec) { cudaGraphExecDestroy(cache->exec); cache->exec = nullptr; }
          if (cache->graph) { cudaGraphDestroy(cache->graph); cache->graph = nullptr; }
          cache->per_iter = 0;
          break;
        }
        (timed ? cache->graph_timed : cache->graph) = graph;
        (timed ? cache->exec_timed : cache->exec) = exec;
      }

    }
  }
  if (++cache->solves == 2 && cache->exec && !cache->exec_chunk && niter > kChunk) capture_chunk(cache, s);
  for (; it < niter; ++it) {
    if (cancel && cancel->load()) break;
    // whole chunks while they fit before the last iteration (which replays
    // the instrumented copy when stage timing is on)
    if (cache->exec_chunk && it + kChunk + (cache->exec_timed ? 1 : 0) <= niter) {
      cudaError_t ce = cudaGraphLaunch(cache->exec_chunk, s);
      if (ce != cudaSuccess) {
        cudaGetLastError();
        A->pcg_cache.reset();
        return set_error(PG_CUDA_ERROR, "graph launch: %s", cudaGetErrorString(ce));
      }
      count_launch(kChunk * cache->per_iter);
      it += kChunk - 1;
      continue;
    }
    if (cache->exec) {
      cudaGraphExec_t exec = (cache->exec_timed && it + 1 == niter) ? cache->exec_timed : cache->exec;
      cudaError_t ce = cudaGraphLaunch(exec, s);
      if (ce != cudaSuccess) {
        cudaGetLastError();
        A->pcg_cache.reset();
        return set_error(PG_CUDA_ERROR, "graph launch: %s", cudaGetErrorString(ce));
      }
      count_launch(cache->per_iter);
    } else {
      st = S.iteration(s);
      if (st != PG_OK) { A->pcg_cache.reset(); return st; }
    }
  }
  PG_CUDA(cudaMemcpyAsync(xout, S.x.p, ni * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  if (iters_dev) PG_LAUNCH(k_copy_iters, 1, 32, 0, s, S.fl.p, S.nseg, iters_dev);
  if (cancel && cancel->load()) {
    PG_CUDA(cudaStreamSynchronize(s));
    return set_error(PG_CANCELLED, "solve cancelled");
  }
  return PG_OK;
}

// Gradient / Denom as stand-alone kernels (tests).
__global__ void k_grad_only(PenDev R, const float2* __restrict__ x, float2* __restrict__ g) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < R.N; j += (uint64_t)gridDim.x * blockDim.x)
    g[j] = grad_at(R, x, nullptr, 0.f, j);
}
__global__ void k_denom_only(PenDev R, const float2* __restrict__ ddir, const float2* __restrict__ x, double* part,
                             int nb) {
  double a = 0.0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < R.N; j += (uint64_t)gridDim.x * blockDim.x) {
    for (int dim = 0; dim < R.nd; ++dim) {
      const uint64_t off = R.off[dim];
      if (j < off || off >= R.N) continue;
      const float2 cd = csub(ddir[j], ddir[j - off]);
      const float2 cz = csub(x[j], x[j - off]);
      a += (double)wpot(R, cz) * ((double)cd.x * cd.x + (double)cd.y * cd.y);
    }
  }
  block_store2(a, 0.0, part, nb);
}

// ---------------------------------------------------------------------------
// R_lowRank (lowRank/R_lowRank.cpp:27-95) and the PCG loop that carries it.
//
// With x = vec(X), X N x K, the wrapper penalises the columns of
// I = X * trans(v.cols(0, K-1)) (:42-44; trans is the conjugate transpose, so
// I[:, j] = sum_k X[:, k] conj(v[j + K k])).  Gradient (:50-64) returns
// vectorise(strans(v.cols(0, K-1)) * strans(Y)), Y_j = R.Gradient(I_j): a
// K x N matrix stored k fastest, g[k + K n] = sum_j v[j + K k] Y[n, j].  That
// product is defined only when K == Nimg (a K x K matrix times an Nimg x N
// one), so the wrapper takes a square basis.  Denom (:67-87) is
// R.Beta * sum_j R.Denom(D_j, I_j) with D = Ddir * trans(v), R.Denom already
// carrying one factor beta.
// ---------------------------------------------------------------------------
__global__ void k_grad_images(PenDev R, int K, const float2* __restrict__ x, float2* __restrict__ g) {
  const uint64_t n = R.N * (uint64_t)K;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t img = t / R.N, j = t - img * R.N;
    g[t] = grad_at(R, x + img * R.N, nullptr, 0.f, j);
  }
}

__global__ void k_denom_images(PenDev R, int K, const float2* __restrict__ ddir, const float2* __restrict__ x,
                               double* part, int nb) {
  double a = 0.0;
  const uint64_t n = R.N * (uint64_t)K;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t img = t / R.N, j = t - img * R.N;
    const float2* di = ddir + img * R.N;
    const float2* xi = x + img * R.N;
    for (int dim = 0; dim < R.nd; ++dim) {
      const uint64_t off = R.off[dim];
      if (j < off || off >= R.N) continue;
      const float2 cd = csub(di[j], di[j - off]);
      const float2 cz = csub(xi[j], xi[j - off]);
      a += (double)wpot(R, cz) * ((double)cd.x * cd.x + (double)cd.y * cd.y);
    }
  }
  block_store2(a, 0.0, part, nb);
}

// Block partials of a stand-alone reduction, added on the host in block order.
struct HostSums {
  DevBuf<double> part;
  std::vector<double> h;
  pg_status fetch(int nb, double* s0, double* s1, cudaStream_t s) {
    h.resize(2 * (size_t)nb);
    PG_CUDA(cudaMemcpyAsync(h.data(), part.p, 2 * (size_t)nb * sizeof(double), cudaMemcpyDeviceToHost, s));
    PG_CUDA(cudaStreamSynchronize(s));
    double a = 0.0, b = 0.0;
    for (int i = 0; i < nb; ++i) { a += h[i]; b += h[nb + i]; }
    if (s0) *s0 = a;
    if (s1) *s1 = b;
    return PG_OK;
  }
};

struct LowRankPen {
  PenDev R;
  double beta = 0;
  int K = 1;
  DevBuf<float2> cr;    // K x K, cr[j + K k] = conj(v[j + K k]): the mixing into I
  DevBuf<float2> cg;    // K x K, cg[k + K j] = v[j + K k]: the gradient's strans(v)
  DevBuf<float2> I, D, Y;
  HostSums sums;

  pg_status init(const pg_penalty& Rh, uint64_t rank, const float* v, cudaStream_t s) {
    R = make_pen(Rh);
    beta = Rh.beta;
    K = (int)rank;
    const float2* vb = reinterpret_cast<const float2*>(v);
    std::vector<float2> hr(rank * rank), hg(rank * rank);
    for (uint64_t j = 0; j < rank; ++j)
      for (uint64_t k = 0; k < rank; ++k) {
        const float2 e = vb[j + rank * k];
        hr[j + rank * k] = make_float2(e.x, -e.y);
        hg[k + rank * j] = e;
      }
    PG_TRY(cr.upload(hr.data(), hr.size(), s));
    PG_TRY(cg.upload(hg.data(), hg.size(), s));
    PG_TRY(I.alloc(R.N * rank));
    PG_TRY(D.alloc(R.N * rank));
    PG_TRY(Y.alloc(R.N * rank));
    return PG_OK;
  }
  pg_status gradient(const float2* x, float2* g, cudaStream_t s) {
    PG_TRY(mix_columns(R.N, K, K, x, cr.p, false, I.p, s));
    PG_LAUNCH(k_grad_images, (unsigned)red_blocks(R.N * K), kRed, 0, s, R, K, I.p, Y.p);
    return mix_columns(R.N, K, K, Y.p, cg.p, true, g, s);
  }
  pg_status denom(const float2* ddir, const float2* x, double* out, cudaStream_t s) {
    PG_TRY(mix_columns(R.N, K, K, x, cr.p, false, I.p, s));
    PG_TRY(mix_columns(R.N, K, K, ddir, cr.p, false, D.p, s));
    const int nb = red_blocks(R.N * K);
    PG_TRY(sums.part.alloc(2 * (uint64_t)nb));
    PG_LAUNCH(k_denom_images, (unsigned)nb, kRed, 0, s, R, K, D.p, I.p, sums.part.p, nb);
    double a = 0.0;
    PG_TRY(sums.fetch(nb, &a, nullptr, s));
    *out = a * beta * beta;
    return PG_OK;
  }
};

pg_status lowrank_penalty_check(const pg_penalty& Rh, uint64_t rank, uint64_t n_img) {
  if (rank == 0 || rank > 1024) return set_error(PG_INVALID_ARG, "R_lowRank: rank %llu", (unsigned long long)rank);
  if (n_img != rank)
    return set_error(PG_INVALID_ARG,
                     "R_lowRank: the gradient multiplies strans(v.cols(0, rank-1)) (%llux%llu) by an %llu x N "
                     "matrix, defined only when rank == the number of images",
                     (unsigned long long)rank, (unsigned long long)rank, (unsigned long long)n_img);
  if (Rh.kind != PG_PENALTY_QUAD && Rh.kind != PG_PENALTY_TV) return set_error(PG_INVALID_ARG, "unknown penalty");
  if (Rh.kind == PG_PENALTY_TV && !(Rh.delta > 0)) return set_error(PG_INVALID_ARG, "TV penalty needs delta > 0");
  return PG_OK;
}

// ---- the PCG loop with the low-rank wrapper ---------------------------------
// solve_pwls_pcg (solve_pwls_pcg.hpp:48-167) over LRobj with R_lowRank.  The
// wrapper's gradient mixes the K images (not a local stencil), so the
// penalty terms are separate passes (mix, per-image stencil, mix); the
// scalars stay on the device as in the fused solver (FP64 last-block sums,
// early-exit flags), so an iteration has no host step and is replayed as
// one CUDA graph.  The kernels shared with the fused solver run with one
// segment.

// ngrad = A'r - pgrad; partials |A'r|^2 and |ngrad|^2; then the early exit on
// a vanishing gradient (:88-91) and the CG coefficient (:95-110).
__global__ void k_lr_ngrad(uint64_t n, float2* __restrict__ ngrad, const float2* __restrict__ pgrad, double* part,
                           int nb, unsigned* counter, double* sc, uint32_t* fl) {
  if (fl[F_DONE]) return;
  double a = 0.0, b = 0.0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const float2 raw = ngrad[j];
    a += (double)raw.x * raw.x + (double)raw.y * raw.y;
    const float2 v = csub(raw, pgrad[j]);
    ngrad[j] = v;
    b += (double)v.x * v.x + (double)v.y * v.y;
  }
  block_store2(a, b, part, nb);
  if (!last_block(counter)) return;
  const double gn = block_part_sum(part, nb, 0);
  const double nw = block_part_sum(part, nb, 1);
  if (threadIdx.x == 0) {
    if (sqrt(gn) / sc[S_YWY] < 1e-10) { fl[F_DONE] = 1; fl[F_REASON] = 1; return; }
    double gamma = 0.0;
    if (fl[F_IT] > 0) gamma = (fabs(sc[S_OLD]) < 1e-10) ? 0.0 : nw / sc[S_OLD];
    sc[S_GAMMA] = gamma;
    sc[S_OLD] = nw;
  }
}

// xs = x + step ddir: the point of a Newton step (:133).
__global__ void k_lr_point(uint64_t n, const float2* __restrict__ x, const float2* __restrict__ ddir,
                           float2* __restrict__ xs, const double* sc, const uint32_t* fl) {
  if (fl[F_DONE]) return;
  const float st = (float)sc[S_STEP];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float2 u = x[i], v = ddir[i];
    xs[i] = make_float2(u.x + st * v.x, u.y + st * v.y);
  }
}

// R_lowRank Denom (R_lowRank.cpp:67-87) over the mixed images D (of ddir) and
// I (of xs): beta^2 sum_j sum_dims wpot(Cd I_j) |Cd D_j|^2; then the Newton
// denominator dAWAd + pdenom and its range test (:136-140).
__global__ void k_lr_denom(PenDev R, int K, const float2* __restrict__ D, const float2* __restrict__ I, double beta,
                           double* part, int nb, unsigned* counter, double* sc, uint32_t* fl) {
  if (fl[F_DONE]) return;
  double a = 0.0;
  const uint64_t n = R.N * (uint64_t)K;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t img = t / R.N, j = t - img * R.N;
    const float2* di = D + img * R.N;
    const float2* xi = I + img * R.N;
    for (int dim = 0; dim < R.nd; ++dim) {
      const uint64_t off = R.off[dim];
      if (j < off || off >= R.N) continue;
      const float2 cd = csub(di[j], di[j - off]);
      const float2 cz = csub(xi[j], xi[j - off]);
      a += (double)wpot(R, cz) * ((double)cd.x * cd.x + (double)cd.y * cd.y);
    }
  }
  block_store2(a, 0.0, part, nb);
  if (!last_block(counter)) return;
  const double pd = block_part_sum(part, nb, 0);
  if (threadIdx.x == 0) {
    const double denom = sc[S_DAWAD] + pd * beta * beta;
    if (fabs(denom) < 1e-20 || fabs(denom) > 1e25) { fl[F_DONE] = 1; fl[F_REASON] = 3; return; }
    sc[S_PDEN] = denom;
  }
}

// pdot = Re<ddir, Gradient(xs)>; step -= (-dAWr + step dAWAd + pdot) / denom (:141-149).
__global__ void k_lr_step(uint64_t n, const float2* __restrict__ ddir, const float2* __restrict__ pgrad, double* part,
                          int nb, unsigned* counter, double* sc, uint32_t* fl) {
  if (fl[F_DONE]) return;
  double b = 0.0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float2 u = ddir[i], v = pgrad[i];
    b += (double)u.x * v.x + (double)u.y * v.y;
  }
  block_store2(b, 0.0, part, nb);
  if (!last_block(counter)) return;
  const double pdot = block_part_sum(part, nb, 0);
  if (threadIdx.x == 0) {
    const double step = sc[S_STEP];
    sc[S_STEP] = step - (-sc[S_DAWR] + step * sc[S_DAWAD] + pdot) / sc[S_PDEN];
  }
}

// Buffers, penalty and the captured iteration of low-rank solves, cached on
// the LRobj operator.  A new solve with the same penalty shape re-uploads the
// basis into the same device matrices and replays the graph.
struct LowRankCache : pg_pcg_cache_base {
  LowRankPen P;
  pg_penalty R{};
  uint64_t rank = 0;
  bool w_ones = true;
  uint64_t prof_epoch = 0;
  DevBuf<float2> x, Ax, r, ngrad, pgrad, ddir, Adir, xs, ybuf;
  DevBuf<float> wbuf;
  DevBuf<double> part, sc;
  DevBuf<uint32_t> fl;
  DevBuf<unsigned> counter;
  int nbd = 1, nbi = 1, nbk = 1;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t per_iter = 0;
  ~LowRankCache() override {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
  bool matches(const pg_penalty& q, uint64_t k, bool ones) const {
    return R.kind == q.kind && R.nx == q.nx && R.ny == q.ny && R.nz == q.nz && R.beta == q.beta &&
           R.delta == q.delta && R.dims2penalize == q.dims2penalize && rank == k && w_ones == ones &&
           prof_epoch == g_profile_epoch;
  }

  // One iteration; r = W (.) (y - Ax) holds on entry and on exit.
  pg_status iteration(pg_op_s* A, cudaStream_t s) {
    const uint64_t ni = A->n_image, nd = A->n_data;
    const int pst = 0;   // one segment
    PG_TRY(A->adjoint(r.p, ngrad.p, s));
    PG_TRY(P.gradient(x.p, pgrad.p, s));
    PG_LAUNCH(k_lr_ngrad, (unsigned)nbi, kRed, 0, s, ni, ngrad.p, pgrad.p, part.p, nbi, counter.p, sc.p, fl.p);
    PG_LAUNCH(k_ddir, (unsigned)nbi, kRed, 0, s, ni, ngrad.p, ddir.p, part.p, nbi, counter.p, sc.p, fl.p, pst);
    PG_TRY(A->forward(ddir.p, Adir.p, s));
    PG_LAUNCH(k_daw, (unsigned)nbd, kRed, 0, s, nd, Adir.p, wbuf.p, r.p, part.p, nbd, counter.p, sc.p, fl.p, 0, 0.0,
              pst);
    for (int k = 0; k < 3; ++k) {                                    // :128-150
      PG_LAUNCH(k_lr_point, (unsigned)nbi, kRed, 0, s, ni, x.p, ddir.p, xs.p, sc.p, fl.p);
      PG_TRY(mix_columns(P.R.N, P.K, P.K, xs.p, P.cr.p, false, P.I.p, s));
      PG_TRY(mix_columns(P.R.N, P.K, P.K, ddir.p, P.cr.p, false, P.D.p, s));
      PG_LAUNCH(k_lr_denom, (unsigned)nbk, kRed, 0, s, P.R, P.K, P.D.p, P.I.p, P.beta, part.p, nbk, counter.p, sc.p,
                fl.p);
      PG_TRY(P.gradient(xs.p, pgrad.p, s));
      PG_LAUNCH(k_lr_step, (unsigned)nbi, kRed, 0, s, ni, ddir.p, pgrad.p, part.p, nbi, counter.p, sc.p, fl.p);
    }
    PG_LAUNCH(k_update, (unsigned)red_blocks(std::max(nd, ni)), kRed, 0, s, ni, nd, x.p, ddir.p, Ax.p, Adir.p, ybuf.p,
              wbuf.p, r.p, sc.p, fl.p);
    return PG_OK;
  }
};

pg_status make_lowrank_cache(pg_op_s* A, const pg_penalty& Rh, uint64_t rank, const float* v, bool w_ones,
                             std::unique_ptr<LowRankCache>* out, cudaStream_t s) {
  auto c = std::make_unique<LowRankCache>();
  const uint64_t ni = A->n_image, nd = A->n_data;
  PG_TRY(c->P.init(Rh, rank, v, s));
  c->R = Rh;
  c->rank = rank;
  c->w_ones = w_ones;
  c->prof_epoch = g_profile_epoch;
  c->nbd = red_blocks(nd);
  c->nbi = red_blocks(ni);
  c->nbk = red_blocks(c->P.R.N * rank);
  for (DevBuf<float2>* b : {&c->x, &c->ngrad, &c->pgrad, &c->ddir, &c->xs}) PG_TRY(b->alloc(ni));
  for (DevBuf<float2>* b : {&c->Ax, &c->r, &c->Adir, &c->ybuf}) PG_TRY(b->alloc(nd));
  PG_TRY(c->wbuf.alloc(nd));
  if (w_ones) PG_LAUNCH(k_fill_ones, ceil_div(nd, 256), 256, 0, s, nd, c->wbuf.p);
  PG_TRY(c->part.alloc(2 * (uint64_t)std::max(c->nbd, std::max(c->nbi, c->nbk))));
  PG_TRY(c->sc.alloc(S_NSCAL));
  PG_TRY(c->fl.alloc(F_NFLAG));
  PG_TRY(c->counter.alloc(1));
  PG_CUDA(cudaMemsetAsync(c->counter.p, 0, sizeof(unsigned), s));
  *out = std::move(c);
  return PG_OK;
}

pg_status pcg_solve_lowrank(pg_op_s* A, const pg_penalty& Rh, uint64_t rank, const float* v, const float2* x0,
                            const float* W, const float2* y, uint64_t niter, float2* xout, uint64_t* iters,
                            cudaStream_t s) {
  const uint64_t ni = A->n_image, nd = A->n_data;
  auto* c = dynamic_cast<LowRankCache*>(A->pcg_cache.get());
  if (!c || !c->matches(Rh, rank, W == nullptr)) {
    A->pcg_cache.reset();
    std::unique_ptr<LowRankCache> nc;
    PG_TRY(make_lowrank_cache(A, Rh, rank, v, W == nullptr, &nc, s));
    c = nc.get();
    A->pcg_cache = std::move(nc);
  } else {
    PG_TRY(c->P.init(Rh, rank, v, s));   // same shapes: the graph's matrices, rewritten in place
  }
  // inputs into the buffers the graph reads
  PG_CUDA(cudaMemcpyAsync(c->ybuf.p, y, nd * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  if (W) PG_CUDA(cudaMemcpyAsync(c->wbuf.p, W, nd * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if (x0) PG_CUDA(cudaMemcpyAsync(c->x.p, x0, ni * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  else PG_CUDA(cudaMemsetAsync(c->x.p, 0, ni * sizeof(float2), s));
  PG_CUDA(cudaMemsetAsync(c->ddir.p, 0, ni * sizeof(float2), s));
  pg_status st = PG_OK;
  if (x0) st = A->forward(c->x.p, c->Ax.p, s);                       // :55
  else PG_CUDA(cudaMemsetAsync(c->Ax.p, 0, nd * sizeof(float2), s));   // A * 0 = 0 exactly
  if (st != PG_OK) { A->pcg_cache.reset(); return st; }
  PG_LAUNCH(k_ywy, (unsigned)c->nbd, kRed, 0, s, nd, c->ybuf.p, c->wbuf.p, c->part.p, c->nbd, 0);
  PG_LAUNCH(k_scalar_init, 1, 32, 0, s, c->part.p, c->nbd, 0, c->sc.p, c->fl.p);
  PG_LAUNCH(k_residual, (unsigned)c->nbd, kRed, 0, s, nd, c->ybuf.p, c->Ax.p, c->wbuf.p, c->r.p);
  uint64_t it = 0;
  if (!c->exec && niter > 0) {
    // the first iteration eagerly (it sizes every workspace), then one capture
    st = c->iteration(A, s);
    if (st != PG_OK) { A->pcg_cache.reset(); return st; }
    it = 1;
    if (graphs_enabled() && niter > 1) {
      const uint64_t before = g_launches.load();
      g_profile_suppress = true;
      PG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      st = c->iteration(A, s);
      cudaGraph_t graph = nullptr;
      cudaError_t ce = cudaStreamEndCapture(s, &graph);
      g_profile_suppress = false;
      c->per_iter = g_launches.load() - before;
      g_launches.fetch_sub(c->per_iter);
      if (st != PG_OK) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        A->pcg_cache.reset();
        return st;
      }
      cudaGraphExec_t exec = nullptr;
      if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
      if (ce == cudaSuccess) {
        c->graph = graph;
        c->exec = exec;
      } else {
        // nothing captured ran: continue from the eager iteration without graphs
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        c->per_iter = 0;
      }
    }
  }
  for (; it < niter; ++it) {
    if (c->exec) {
      cudaError_t ce = cudaGraphLaunch(c->exec, s);
      if (ce != cudaSuccess) {
        cudaGetLastError();
        A->pcg_cache.reset();
        return set_error(PG_CUDA_ERROR, "graph launch: %s", cudaGetErrorString(ce));
      }
      count_launch(c->per_iter);
    } else {
      st = c->iteration(A, s);
      if (st != PG_OK) { A->pcg_cache.reset(); return st; }
    }
  }
  PG_CUDA(cudaMemcpyAsync(xout, c->x.p, ni * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  uint32_t done = 0;
  PG_CUDA(cudaMemcpyAsync(&done, c->fl.p + F_COMPLETED, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  if (iters) *iters = done;
  return PG_OK;
}

}  // namespace pg

using namespace pg;

extern "C" {

pg_status pg_pcg_solve_device(pg_op A, const void* x0, const void* W, const void* y, const pg_penalty* R,
                              uint64_t niter, void* x_out, void* iters_done_dev, void* stream) {
  if (!A || !y || !R || !x_out) return set_error(PG_INVALID_ARG, "pcg: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  return pcg_solve_device(A, (const float2*)x0, (const float*)W, (const float2*)y, *R, niter, (float2*)x_out,
                          (uint32_t*)iters_done_dev, s);
}

pg_status pg_pcg_solve(pg_op A, const float* x0, const float* W, const float* y, const pg_penalty* R, uint64_t niter,
                       float* x_out, uint64_t* iters_done) {
  if (!A || !y || !R || !x_out) return set_error(PG_INVALID_ARG, "pcg: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  // the operator's staging buffers: no device allocation after the first call
  PG_TRY(A->hy.upload(reinterpret_cast<const float2*>(y), A->n_data, s));
  if (x0) PG_TRY(A->hx0.upload(reinterpret_cast<const float2*>(x0), A->n_image, s));
  if (W) PG_TRY(A->hw.upload(W, A->n_data, s));
  PG_TRY(A->hx.alloc(A->n_image));
  PG_TRY(A->hit.alloc(A->n_seg ? A->n_seg : 1));   // one count per segment; the first is reported
  PG_TRY(pcg_solve_device(A, x0 ? A->hx0.p : nullptr, W ? A->hw.p : nullptr, A->hy.p, *R, niter, A->hx.p, A->hit.p,
                          s));
  PG_CUDA(cudaMemcpyAsync(x_out, A->hx.p, A->n_image * sizeof(float2), cudaMemcpyDeviceToHost, s));
  uint32_t n = 0;
  PG_CUDA(cudaMemcpyAsync(&n, A->hit.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  if (iters_done) *iters_done = n;
  return PG_OK;
}

pg_status pg_recon_solve(pg_op Sg, const pg_penalty* R, const float* data, uint64_t niter, float* image_out) {
  // reconSolve.h:63-82: W = ones, x0 = zeros.
  return pg_pcg_solve(Sg, nullptr, nullptr, data, R, niter, image_out, nullptr);
}

pg_status pg_penalty_gradient_device(const pg_penalty* R, const void* x, void* g, void* stream) {
  if (!R || !x || !g) return set_error(PG_INVALID_ARG, "penalty: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  PenDev P = make_pen(*R);
  PG_LAUNCH(k_grad_only, (unsigned)red_blocks(P.N), kRed, 0, s, P, (const float2*)x, (float2*)g);
  return PG_OK;
}

// ---- checkpoint / resume ----------------------------------------------------
// The solver state between iterations, as a host blob: a header, then x, Ax,
// the residual r and the direction (ni, nd, nd, ni complex), the previous
// direction for the quadratic penalty (ni), the FP64 scalars and the flags.
// The blob records the objective it was computed for (operator shape and
// penalty parameters); loading it for another objective is refused, since the
// saved direction and FP64 scalars belong to the saved one.
struct PcgStateHeader {
  char magic[8];
  uint64_t ni, nd;
  int32_t kind, has_prev;
  uint64_t nscal, nflag;
  uint64_t nx, ny, nz, dims2penalize;
  float beta, delta;
};
constexpr char kStateMagic[9] = "PGPCGST2";

static uint64_t state_bytes(uint64_t ni, uint64_t nd, bool prev) {
  return sizeof(PcgStateHeader) + (2 * ni + 2 * nd + (prev ? ni : 0)) * sizeof(float2) + S_NSCAL * sizeof(double) +
         F_NFLAG * sizeof(uint32_t);
}

pg_status pg_pcg_state_size(pg_op A, uint64_t* bytes) {
  if (!A || !bytes) return set_error(PG_INVALID_ARG, "pcg state: null argument");
  auto* c = dynamic_cast<PcgCache*>(A->pcg_cache.get());
  if (!c) return set_error(PG_INVALID_ARG, "pcg state: no solve has run on this operator");
  if (c->S.nseg > 1) return set_error(PG_INVALID_ARG, "pcg state: operators of several segments are not saved");
  *bytes = state_bytes(A->n_image, A->n_data, c->S.ddir_prev.p != nullptr);
  return PG_OK;
}

pg_status pg_pcg_state_save(pg_op A, void* host, uint64_t bytes) {
  uint64_t need = 0;
  PG_TRY(pg_pcg_state_size(A, &need));
  if (!host || bytes < need) return set_error(PG_INVALID_ARG, "pcg state: buffer of %llu bytes, %llu needed",
                                              (unsigned long long)bytes, (unsigned long long)need);
  auto* c = dynamic_cast<PcgCache*>(A->pcg_cache.get());
  Solver& S = c->S;
  PG_CUDA(cudaDeviceSynchronize());   // the solve may have run on any stream
  PcgStateHeader h{};
  std::memcpy(h.magic, kStateMagic, 8);
  h.ni = A->n_image;
  h.nd = A->n_data;
  h.kind = S.R.kind;
  h.nx = c->R.nx;
  h.ny = c->R.ny;
  h.nz = c->R.nz;
  h.dims2penalize = c->R.dims2penalize;
  h.beta = c->R.beta;
  h.delta = c->R.delta;
  h.has_prev = S.ddir_prev.p ? 1 : 0;
  h.nscal = S_NSCAL;
  h.nflag = F_NFLAG;
  char* o = static_cast<char*>(host);
  std::memcpy(o, &h, sizeof(h));
  o += sizeof(h);
  auto take = [&](const void* d, uint64_t nb) -> pg_status {
    PG_CUDA(cudaMemcpy(o, d, nb, cudaMemcpyDeviceToHost));
    o += nb;
    return PG_OK;
  };
  PG_TRY(take(S.x.p, h.ni * sizeof(float2)));
  PG_TRY(take(S.Ax.p, h.nd * sizeof(float2)));
  PG_TRY(take(S.r.p, h.nd * sizeof(float2)));
  PG_TRY(take(S.ddir.p, h.ni * sizeof(float2)));
  if (h.has_prev) PG_TRY(take(S.ddir_prev.p, h.ni * sizeof(float2)));
  PG_TRY(take(S.sc.p, S_NSCAL * sizeof(double)));
  PG_TRY(take(S.fl.p, F_NFLAG * sizeof(uint32_t)));
  return PG_OK;
}

pg_status pg_pcg_state_load(pg_op A, const pg_penalty* R, const void* host, uint64_t bytes) {
  if (!A || !R || !host) return set_error(PG_INVALID_ARG, "pcg state: null argument");
  if (A->n_seg > 1) return set_error(PG_INVALID_ARG, "pcg state: operators of several segments are not loaded");
  PcgStateHeader h{};
  if (bytes < sizeof(h)) return set_error(PG_INVALID_ARG, "pcg state: %llu bytes", (unsigned long long)bytes);
  std::memcpy(&h, host, sizeof(h));
  if (std::memcmp(h.magic, kStateMagic, 8) != 0 || h.nscal != S_NSCAL || h.nflag != F_NFLAG)
    return set_error(PG_INVALID_ARG, "pcg state: not a solver state of this library");
  if (h.ni != A->n_image || h.nd != A->n_data || h.kind != R->kind ||
      (h.has_prev != 0) != (R->kind == PG_PENALTY_QUAD) || bytes < state_bytes(h.ni, h.nd, h.has_prev != 0))
    return set_error(PG_INVALID_ARG, "pcg state: saved for a %llux%llu operator with penalty %d",
                     (unsigned long long)h.nd, (unsigned long long)h.ni, h.kind);
  if (R->nx * R->ny * R->nz != A->n_image) return set_error(PG_INVALID_ARG, "pcg state: penalty size");
  if (h.nx != R->nx || h.ny != R->ny || h.nz != R->nz || h.dims2penalize != R->dims2penalize || h.beta != R->beta ||
      (R->kind == PG_PENALTY_TV && h.delta != R->delta))
    return set_error(PG_INVALID_ARG,
                     "pcg state: saved for penalty %llux%llux%llu beta %g delta %g dims %llu, not this one",
                     (unsigned long long)h.nx, (unsigned long long)h.ny, (unsigned long long)h.nz, (double)h.beta,
                     (double)h.delta, (unsigned long long)h.dims2penalize);
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  A->pcg_cache.reset();
  std::unique_ptr<PcgCache> c;
  PG_TRY(make_cache(A, *R, true, &c, s));
  Solver& S = c->S;
  const char* i = static_cast<const char*>(host) + sizeof(h);
  auto put = [&](void* d, uint64_t nb) -> pg_status {
    PG_CUDA(cudaMemcpyAsync(d, i, nb, cudaMemcpyHostToDevice, s));
    i += nb;
    return PG_OK;
  };
  PG_TRY(put(S.x.p, h.ni * sizeof(float2)));
  PG_TRY(put(S.Ax.p, h.nd * sizeof(float2)));
  PG_TRY(put(S.r.p, h.nd * sizeof(float2)));
  PG_TRY(put(S.ddir.p, h.ni * sizeof(float2)));
  if (h.has_prev) PG_TRY(put(S.ddir_prev.p, h.ni * sizeof(float2)));
  PG_TRY(put(S.sc.p, S_NSCAL * sizeof(double)));
  PG_TRY(put(S.fl.p, F_NFLAG * sizeof(uint32_t)));
  PG_CUDA(cudaStreamSynchronize(s));
  A->pcg_cache = std::move(c);
  return PG_OK;
}

pg_status pg_pcg_resume_device(pg_op A, const void* W, const void* y, const pg_penalty* R, uint64_t niter,
                               void* x_out, void* iters_done_dev, void* stream) {
  if (!A || !y || !R || !x_out) return set_error(PG_INVALID_ARG, "pcg resume: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  return pcg_solve_device(A, nullptr, (const float*)W, (const float2*)y, *R, niter, (float2*)x_out,
                          (uint32_t*)iters_done_dev, s, nullptr, true);
}

pg_status pg_pcg_resume(pg_op A, const float* W, const float* y, const pg_penalty* R, uint64_t niter, float* x_out,
                        uint64_t* iters_done) {
  if (!A || !y || !R || !x_out) return set_error(PG_INVALID_ARG, "pcg resume: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  PG_TRY(A->hy.upload(reinterpret_cast<const float2*>(y), A->n_data, s));
  if (W) PG_TRY(A->hw.upload(W, A->n_data, s));
  PG_TRY(A->hx.alloc(A->n_image));
  PG_TRY(A->hit.alloc(1));
  PG_TRY(pcg_solve_device(A, nullptr, W ? A->hw.p : nullptr, A->hy.p, *R, niter, A->hx.p, A->hit.p, s, nullptr,
                          true));
  PG_CUDA(cudaMemcpyAsync(x_out, A->hx.p, A->n_image * sizeof(float2), cudaMemcpyDeviceToHost, s));
  uint32_t n = 0;
  PG_CUDA(cudaMemcpyAsync(&n, A->hit.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  if (iters_done) *iters_done = n;
  return PG_OK;
}

pg_status pg_pcg_solve_lowrank_device(pg_op A, const void* x0, const void* W, const void* y, const pg_penalty* R,
                                      uint64_t rank, uint64_t n_img, const float* v, uint64_t niter, void* x_out,
                                      uint64_t* iters_done, void* stream) {
  if (!A || !y || !R || !v || !x_out) return set_error(PG_INVALID_ARG, "low-rank pcg: null argument");
  PG_TRY(lowrank_penalty_check(*R, rank, n_img));
  if (R->nx * R->ny * R->nz * rank != A->n_image)
    return set_error(PG_INVALID_ARG, "low-rank pcg: penalty %llux%llux%llu x rank %llu does not match the model's %llu",
                     (unsigned long long)R->nx, (unsigned long long)R->ny, (unsigned long long)R->nz,
                     (unsigned long long)rank, (unsigned long long)A->n_image);
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  return pcg_solve_lowrank(A, *R, rank, v, (const float2*)x0, (const float*)W, (const float2*)y, niter,
                           (float2*)x_out, iters_done, s);
}

pg_status pg_pcg_solve_lowrank(pg_op A, const float* x0, const float* W, const float* y, const pg_penalty* R,
                               uint64_t rank, uint64_t n_img, const float* v, uint64_t niter, float* x_out,
                               uint64_t* iters_done) {
  if (!A || !y || !R || !v || !x_out) return set_error(PG_INVALID_ARG, "low-rank pcg: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  PG_TRY(A->hy.upload(reinterpret_cast<const float2*>(y), A->n_data, s));
  if (x0) PG_TRY(A->hx0.upload(reinterpret_cast<const float2*>(x0), A->n_image, s));
  if (W) PG_TRY(A->hw.upload(W, A->n_data, s));
  PG_TRY(A->hx.alloc(A->n_image));
  PG_TRY(pg_pcg_solve_lowrank_device(A, x0 ? A->hx0.p : nullptr, W ? A->hw.p : nullptr, A->hy.p, R, rank, n_img, v,
                                     niter, A->hx.p, iters_done, s));
  PG_CUDA(cudaMemcpyAsync(x_out, A->hx.p, A->n_image * sizeof(float2), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

pg_status pg_lowrank_penalty_gradient_device(const pg_penalty* R, uint64_t rank, uint64_t n_img, const float* v,
                                             const void* x, void* g, void* stream) {
  if (!R || !v || !x || !g) return set_error(PG_INVALID_ARG, "R_lowRank: null argument");
  PG_TRY(lowrank_penalty_check(*R, rank, n_img));
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  LowRankPen P;
  PG_TRY(P.init(*R, rank, v, s));
  PG_TRY(P.gradient((const float2*)x, (float2*)g, s));
  PG_CUDA(cudaStreamSynchronize(s));   // P's buffers are freed on return
  return PG_OK;
}

pg_status pg_lowrank_penalty_denom_device(const pg_penalty* R, uint64_t rank, uint64_t n_img, const float* v,
                                          const void* ddir, const void* x, double* out_host) {
  if (!R || !v || !x || !ddir || !out_host) return set_error(PG_INVALID_ARG, "R_lowRank: null argument");
  PG_TRY(lowrank_penalty_check(*R, rank, n_img));
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  LowRankPen P;
  PG_TRY(P.init(*R, rank, v, s));
  return P.denom((const float2*)ddir, (const float2*)x, out_host, s);
}

pg_status pg_penalty_denom_device(const pg_penalty* R, const void* ddir, const void* x, double* out_host) {
  if (!R || !x || !ddir || !out_host) return set_error(PG_INVALID_ARG, "penalty: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  PenDev P = make_pen(*R);
  const int nb = red_blocks(P.N);
  DevBuf<double> part;
  PG_TRY(part.alloc(2 * (uint64_t)nb));
  PG_LAUNCH(k_denom_only, (unsigned)nb, kRed, 0, s, P, (const float2*)ddir, (const float2*)x, part.p, nb);
  std::vector<double> h(nb);
  PG_CUDA(cudaMemcpyAsync(h.data(), part.p, nb * sizeof(double), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  double a = 0;
  for (double v : h) a += v;
  *out_host = a * R->beta;
  return PG_OK;
}

}  // extern "C"
