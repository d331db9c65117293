// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// extern "C" entry points into the reference's own compiled kernels
// (PowerGrid/gridding.cpp, griddingSupport.cpp, ftCpu.cpp, fftCPU.cpp built in
// place by oracle/Makefile into oracle/_ref/libpgref.so).  Each wrapper
// allocates the scratch buffers the way Gnufft's constructor does
// (Gnufft.cpp:104-113) and calls the reference template exactly as
// Gnufft::operator* / operator/ do (Gnufft.cpp:167-171, 203-207), as the
// spatial interpolation methods do (Gnufft.cpp:238-253, 286-327) and as
// Gdft does (Gdft.cpp:78-80, 120-122).  Nothing here re-implements the math.
#include "gridding.h"
#include "ftCpu.h"
#include "ftCpuWithGrads.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace {

template <typename T>
unsigned long long grid_elems(T gridos, unsigned long long Nx, unsigned long long Ny, unsigned long long Nz) {
  // Gnufft.cpp:55-61
  unsigned long long g = gridos * Nx * gridos * Ny;
  if (Nz > 1) g = g * gridos * Nz;
  return g;
}

template <typename T>
void fd(int M, const T* kx, const T* ky, const T* kz, const T* x, int Nx, int Ny, int Nz, T gridos,
        T kw, T beta, const T* lut, unsigned long long nlut, T* y) {
  const unsigned long long ni = (unsigned long long)Nx * Ny * Nz;
  const unsigned long long ng = grid_elems<T>(gridos, Nx, Ny, Nz);
  std::vector<T> g(2 * ni), gd(2 * ni), gos(2 * ng), gosd(2 * ng), s(2 * (size_t)M);
  computeFd_CPU_Grid<T>(M, kx, ky, kz, x, Nx, Ny, Nz, gridos, kw, beta, lut, nlut, nullptr, nullptr,
                        g.data(), gd.data(), gos.data(), gosd.data(), s.data());
  std::memcpy(y, s.data(), sizeof(T) * 2 * (size_t)M);
}

template <typename T>
void fh(int M, const T* kx, const T* ky, const T* kz, const T* d, int Nx, int Ny, int Nz, T gridos,
        T kw, T beta, const T* lut, unsigned long long nlut, T* x) {
  const unsigned long long ni = (unsigned long long)Nx * Ny * Nz;
  const unsigned long long ng = grid_elems<T>(gridos, Nx, Ny, Nz);
  std::vector<T> g(2 * ni), gd(2 * ni), gos(2 * ng), gosd(2 * ng);
  computeFH_CPU_Grid<T>(M, kx, ky, kz, d, Nx, Ny, Nz, gridos, kw, beta, lut, nlut, nullptr, nullptr,
                        g.data(), gd.data(), gos.data(), gosd.data());
  std::memcpy(x, g.data(), sizeof(T) * 2 * ni);
}

// parameters exactly as Gnufft::forwardSpatialInterp / adjointSpatialInterp
// fill them (Gnufft.cpp:218-236, 266-284)
template <typename T>
parameters<T> interp_params(int M, int Nx, int Ny, int Nz, T gridos, T kw) {
  parameters<T> p;
  p.sync = 0;
  p.binsize = 128;
  p.useLUT = 1;
  p.kernelWidth = kw;
  p.gridOS = gridos;
  p.imageSize[0] = Nx;
  p.imageSize[1] = Ny;
  p.imageSize[2] = Nz;
  p.gridSize[0] = std::ceil(gridos * (T)Nx);
  p.gridSize[1] = std::ceil(gridos * (T)Ny);
  if (p.gridSize[0] % 2) p.gridSize[0] += 1;
  if (p.gridSize[1] % 2) p.gridSize[1] += 1;
  p.gridSize[2] = (Nz == 1) ? Nz : (std::ceil(gridos * (T)Nz));
  p.numSamples = M;
  return p;
}

// forwardSpatialInterp's body (Gnufft.cpp:238-253): samples zeroed, then
// gridding_forward on the caller's grid.
template <typename T>
void ifwd(int M, const T* kx, const T* ky, const T* kz, const T* grid, unsigned long long ngrid, int Nx, int Ny,
          int Nz, T gridos, T kw, T beta, const T* lut, unsigned long long nlut, T* y) {
  parameters<T> p = interp_params<T>(M, Nx, Ny, Nz, gridos, kw);
  std::vector<T> g(grid, grid + 2 * ngrid), s(2 * (size_t)M, (T)0.0);
  if (Nz == 1)
    gridding_forward_2D<T>(M, p, kx, ky, beta, s.data(), lut, nlut, g.data());
  else
    gridding_forward_3D<T>(M, p, kx, ky, kz, beta, s.data(), lut, nlut, g.data());
  std::memcpy(y, s.data(), sizeof(T) * 2 * (size_t)M);
}

// adjointSpatialInterp's body (Gnufft.cpp:286-327): samples packed with
// sdc = 1, grid zeroed, gridding_adjoint.
template <typename T>
void iadj(int M, const T* kx, const T* ky, const T* kz, const T* d, unsigned long long ngrid, int Nx, int Ny,
          int Nz, T gridos, T kw, T beta, const T* lut, unsigned long long nlut, T* grid) {
  parameters<T> p = interp_params<T>(M, Nx, Ny, Nz, gridos, kw);
  std::vector<ReconstructionSample<T>> smp(M);
  for (int i = 0; i < M; ++i) {
    smp[i].kX = kx[i];
    smp[i].kY = ky[i];
    smp[i].kZ = kz[i];
    smp[i].real = d[2 * i];
    smp[i].imag = d[2 * i + 1];
    smp[i].sdc = (T)1.0;
  }
  std::vector<T> g(2 * ngrid, (T)0.0);
  if (Nz == 1)
    gridding_adjoint_2D<T>(M, p, beta, smp.data(), lut, nlut, g.data());
  else
    gridding_adjoint_3D<T>(M, p, beta, smp.data(), lut, nlut, g.data());
  std::memcpy(grid, g.data(), sizeof(T) * 2 * ngrid);
}

}  // namespace

extern "C" {

void pgref_ifwd_f(int M, const float* kx, const float* ky, const float* kz, const float* grid, unsigned long long ng,
                  int Nx, int Ny, int Nz, float os, float kw, float beta, const float* lut, unsigned long long nlut,
                  float* y) {
  ifwd<float>(M, kx, ky, kz, grid, ng, Nx, Ny, Nz, os, kw, beta, lut, nlut, y);
}
void pgref_iadj_f(int M, const float* kx, const float* ky, const float* kz, const float* d, unsigned long long ng,
                  int Nx, int Ny, int Nz, float os, float kw, float beta, const float* lut, unsigned long long nlut,
                  float* grid) {
  iadj<float>(M, kx, ky, kz, d, ng, Nx, Ny, Nz, os, kw, beta, lut, nlut, grid);
}
void pgref_ifwd_d(int M, const double* kx, const double* ky, const double* kz, const double* grid,
                  unsigned long long ng, int Nx, int Ny, int Nz, double os, double kw, double beta, const double* lut,
                  unsigned long long nlut, double* y) {
  ifwd<double>(M, kx, ky, kz, grid, ng, Nx, Ny, Nz, os, kw, beta, lut, nlut, y);
}
void pgref_iadj_d(int M, const double* kx, const double* ky, const double* kz, const double* d,
                  unsigned long long ng, int Nx, int Ny, int Nz, double os, double kw, double beta, const double* lut,
                  unsigned long long nlut, double* grid) {
  iadj<double>(M, kx, ky, kz, d, ng, Nx, Ny, Nz, os, kw, beta, lut, nlut, grid);
}

// calculateLUT (griddingSupport.cpp:52-76); caller frees with pgref_free.
float* pgref_lut_f(float beta, float width, unsigned long long* n) {
  float* lut = nullptr; arma::uword sz = 0;
  calculateLUT<float>(beta, width, lut, sz);
  *n = sz;
  return lut;
}
double* pgref_lut_d(double beta, double width, unsigned long long* n) {
  double* lut = nullptr; arma::uword sz = 0;
  calculateLUT<double>(beta, width, lut, sz);
  *n = sz;
  return lut;
}
void pgref_free(void* p) { free(p); }

void pgref_fd_f(int M, const float* kx, const float* ky, const float* kz, const float* x, int Nx, int Ny,
                int Nz, float os, float kw, float beta, const float* lut, unsigned long long nlut, float* y) {
  fd<float>(M, kx, ky, kz, x, Nx, Ny, Nz, os, kw, beta, lut, nlut, y);
}
void pgref_fh_f(int M, const float* kx, const float* ky, const float* kz, const float* d, int Nx, int Ny,
                int Nz, float os, float kw, float beta, const float* lut, unsigned long long nlut, float* x) {
  fh<float>(M, kx, ky, kz, d, Nx, Ny, Nz, os, kw, beta, lut, nlut, x);
}
void pgref_fd_d(int M, const double* kx, const double* ky, const double* kz, const double* x, int Nx,
                int Ny, int Nz, double os, double kw, double beta, const double* lut, unsigned long long nlut,
                double* y) {
  fd<double>(M, kx, ky, kz, x, Nx, Ny, Nz, os, kw, beta, lut, nlut, y);
}
void pgref_fh_d(int M, const double* kx, const double* ky, const double* kz, const double* d, int Nx,
                int Ny, int Nz, double os, double kw, double beta, const double* lut, unsigned long long nlut,
                double* x) {
  fh<double>(M, kx, ky, kz, d, Nx, Ny, Nz, os, kw, beta, lut, nlut, x);
}

// ftCpu / iftCpu (ftCpu.cpp:95-140, 150-215), planar real/imag like Gdft.cpp:57-96.
void pgref_ft_f(float* kr, float* ki, const float* ir, const float* ii, const float* kx, const float* ky,
                const float* kz, const float* ix, const float* iy, const float* iz, const float* fm,
                const float* t, int nk, int ni) {
  ftCpu<float>(kr, ki, ir, ii, kx, ky, kz, ix, iy, iz, fm, t, nk, ni);
}
void pgref_ift_f(float* ir, float* ii, const float* kr, const float* ki, const float* kx, const float* ky,
                 const float* kz, const float* ix, const float* iy, const float* iz, const float* fm,
                 const float* t, int nk, int ni) {
  iftCpu<float>(ir, ii, kr, ki, kx, ky, kz, ix, iy, iz, fm, t, nk, ni);
}
void pgref_ft_d(double* kr, double* ki, const double* ir, const double* ii, const double* kx,
                const double* ky, const double* kz, const double* ix, const double* iy, const double* iz,
                const double* fm, const double* t, int nk, int ni) {
  ftCpu<double>(kr, ki, ir, ii, kx, ky, kz, ix, iy, iz, fm, t, nk, ni);
}
void pgref_ift_d(double* ir, double* ii, const double* kr, const double* ki, const double* kx,
                 const double* ky, const double* kz, const double* ix, const double* iy, const double* iz,
                 const double* fm, const double* t, int nk, int ni) {
  iftCpu<double>(ir, ii, kr, ki, kx, ky, kz, ix, iy, iz, fm, t, nk, ni);
}

// ftCpuWithGrads / iftCpuWithGrads (ftCpuWithGrads.cpp:93-216), planar like GdftR2.cpp:116-150.
void pgref_ftg_f(float* kr, float* ki, const float* ir, const float* ii, const float* kx, const float* ky,
                 const float* kz, const float* ix, const float* iy, const float* iz, const float* fm, const float* gx,
                 const float* gy, const float* gz, const float* t, int nk, int ni, int nx, int ny, int nz) {
  ftCpuWithGrads<float>(kr, ki, ir, ii, kx, ky, kz, ix, iy, iz, fm, gx, gy, gz, t, nk, ni, nx, ny, nz);
}
void pgref_iftg_f(float* ir, float* ii, const float* kr, const float* ki, const float* kx, const float* ky,
                  const float* kz, const float* ix, const float* iy, const float* iz, const float* fm, const float* gx,
                  const float* gy, const float* gz, const float* t, int nk, int ni, int nx, int ny, int nz) {
  iftCpuWithGrads<float>(ir, ii, kr, ki, kx, ky, kz, ix, iy, iz, fm, gx, gy, gz, t, nk, ni, nx, ny, nz);
}

}  // extern "C"
