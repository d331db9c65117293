// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// extern "C" entry points into the reference's own compiled kernels
// (PowerGrid/gridding.cpp, griddingSupport.cpp, ftCpu.cpp, fftCPU.cpp built in
// place by oracle/Makefile into oracle/_ref/libpgref.so).  Each wrapper
// allocates the scratch buffers the way Gnufft's constructor does
// (Gnufft.cpp:104-113) and calls the reference template exactly as
// Gnufft::operator* / operator/ do (Gnufft.cpp:167-171, 203-207) and as
// Gdft does (Gdft.cpp:78-80, 120-122).  Nothing here re-implements the math.
#include "gridding.h"
#include "ftCpu.h"

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

}  // namespace

extern "C" {

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

}  // extern "C"
