// ORACLE / TEST INFRASTRUCTURE ONLY — the checker, never the product.
//
// CPU restatement of PowerGrid's system-operator path, written for this
// project from the cited reference lines (paths relative to PowerGrid/):
//   Gnufft pipeline     computeFd_CPU_Grid / computeFH_CPU_Grid (gridding.cpp:584-727, 418-581),
//                       gridding_{forward,adjoint}_{2D,3D} (gridding.cpp:31-415),
//                       deapodization/zero_pad/crop/circshift (griddingSupport.cpp:210-627),
//                       LUT + I0 (griddingSupport.cpp:33-76), beta (Gnufft.cpp:84-88)
//   Gdft                ftCpu / iftCpu (ftCpu.cpp:95-215) in float, plus an exact FP64 variant
//   TimeSegmentation    Hanning interpolator (TimeSegmentation.cpp:37-93, 213-218, 252-324)
//   SENSE               SENSE.cpp:33-97
//   pcSenseTimeSeg      pcSenseTimeSeg.cpp:41-171
//   pcSENSE             pcSENSE.cpp:40-153
//   GdftR2              GdftR2.cpp:32-150, ftCpuWithGrads.cpp:76-216
//   spatial interpolation, density compensation   Gnufft.cpp:213-337, reconSupport/directRecon.cpp:28-73
//   Robject/Quad/TV     Robject.cpp:49-193, QuadPenalty.cpp:45-64, TVPenalty.cpp:43-68
//   LRobj, R_lowRank    lowRank/LRobj.cpp:27-68, lowRank/R_lowRank.cpp:27-95
//   solve_pwls_pcg      solve_pwls_pcg.hpp:34-167
//
// Expressions keep the reference's operand types and evaluation order, so
// the float instantiation reproduces the reference CPU path bit for bit when
// both use the same FFT (checked by tests against the reference compiled
// from its own sources).  The double instantiation is the FP64 oracle; for
// the DFT it evaluates sin/cos in double (ftCpu<double> itself calls
// sinf/cosf, ftCpu.cpp:104, 129-130, 203-204).
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <vector>

#include "fft_engine.hpp"

namespace pgo {

using u64 = unsigned long long;

// Single-precision build's pi literal (PGIncludes.h:69): used wherever the
// reference writes MRI_PI, in both instantiations.
constexpr float kPiF = 3.1415926535897932384626433832795029f;
constexpr double kPiD = 3.141592653589793238462643383279502884;  // arma datum::pi

// ---------------------------------------------------------------------------
// Kaiser-Bessel support
// ---------------------------------------------------------------------------

// Modified Bessel I0 by the Abramowitz & Stegun 9.8.1 / 9.8.2 polynomial
// approximations (as tabulated in Numerical Recipes in C, 2nd ed.), with the
// operand types of griddingSupport.cpp:33-48 (double literals, T storage).
template <typename T>
T bessel_i0(T x) {
  T ax = std::abs(x);
  T y;
  T r;
  if (ax < 3.75) {
    y = x / 3.75;
    y = y * y;
    r = 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 +
        y * (0.2659732 + y * (0.360768e-1 + y * 0.45813e-2)))));
  } else {
    y = 3.75 / ax;
    r = (std::exp(ax) / std::sqrt(ax)) *
        (0.39894228 + y * (0.1328592e-1 + y * (0.225319e-2 + y * (-0.157565e-2 +
        y * (0.916281e-2 + y * (-0.2057706e-1 + y * (0.2635537e-1 +
        y * (-0.1647633e-1 + y * 0.392377e-2))))))));
  }
  return r;
}

// LUT[k] = I0(beta*sqrt(1 - k/size))/width, size = 10000*width
// (griddingSupport.cpp:52-76).
template <typename T>
std::vector<T> kb_lut(T beta, T width) {
  std::vector<T> lut;
  if (width > 0) {
    const u64 n = (u64)(10000 * width);
    lut.resize(n);
    for (int k = 0; k < (int)n; ++k) {
      T v = static_cast<T>(k) / static_cast<T>(n);
      lut[k] = bessel_i0<T>(beta * std::sqrt(1.0 - (v))) / width;
    }
  }
  return lut;
}

// Gnufft.cpp:84-88: kernel width 4 and beta from the oversampling factor.
template <typename T>
T kb_beta(T gridos, T width) {
  return kPiF * std::sqrt((gridos - 0.5) * (gridos - 0.5) * (width * width * 4.0) / (gridos * gridos) - 0.8);
}

// ---------------------------------------------------------------------------
// Grid geometry (gridding.cpp:437-446, Gnufft.cpp:55-61)
// ---------------------------------------------------------------------------
template <typename T>
struct Geom {
  int Nx = 1, Ny = 1, Nz = 1;  // image size
  int Gx = 1, Gy = 1, Gz = 1;  // oversampled grid size
  T os = 2;                    // grid oversampling
  T kw = 4;                    // kernel width
  T beta = 0;
  std::vector<T> lut;
  // FP64 evaluation of the float operator (double only): window bounds, LUT
  // index and LUT values as the float instantiation computes them (lut32),
  // every other step in T.  The float and double instantiations pick
  // different LUT entries for some taps, which makes them two operators
  // that differ by ~2e-5; this mode is the float operator without rounding.
  bool float_taps = false;
  std::vector<float> lut32;
  bool is3d() const { return Nz != 1; }
  u64 nimg() const { return (u64)Nx * Ny * Nz; }
  u64 ngrid() const { return (u64)Gx * Gy * Gz; }

  static Geom make(int nx, int ny, int nz, T gridos) {
    Geom g;
    g.Nx = nx; g.Ny = ny; g.Nz = nz; g.os = gridos; g.kw = (T)4.0;
    g.Gx = (int)std::ceil(gridos * (T)nx);
    g.Gy = (int)std::ceil(gridos * (T)ny);
    if (g.Gx % 2) g.Gx += 1;
    if (g.Gy % 2) g.Gy += 1;
    g.Gz = (nz == 1) ? nz : (int)std::ceil(gridos * (T)nz);
    g.beta = kb_beta<T>(gridos, g.kw);
    g.lut = kb_lut<T>(g.beta, g.kw);
    return g;
  }
};

// Window bounds along one axis: clamped to the grid, not wrapped
// (gridding.cpp:67-73).
template <typename T>
inline void window(T s, T kw, T os, int n_image, int& lo, int& hi) {
  lo = (int)(std::max((T)0.0, std::ceil(s - kw * (os) / (T)2.0)));
  hi = (int)(std::min((os * (T)n_image - (T)1.0), std::floor(s + kw * (os) / (T)2.0)));
}

// Nearest-lower LUT entry, zero past the end (gridding.cpp:78-84).
template <typename T>
inline T lut_weight(T s, int n, T os, T kw, const T* lut, u64 nlut) {
  T dist = std::abs(s - ((T)n)) / (os);
  int k0 = (int)((dist * dist * (T)4.0 / (kw * kw)) * (T)nlut);
  if ((u64)k0 >= nlut) return (T)0.0;
  return lut[k0];
}

// Sample position on the grid, window bounds and tap weight through the
// geometry: with float_taps the float operator's values, widened.
template <typename T>
inline T grid_pos(const Geom<T>& g, T k, int n) {
  if (g.float_taps) return (T)((float)g.os * ((float)k + ((float)n) / 2.0f));
  return (g.os) * (k + ((T)n) / (T)2.0);
}
template <typename T>
inline void win(const Geom<T>& g, T s, int n, int& lo, int& hi) {
  if (g.float_taps) window<float>((float)s, (float)g.kw, (float)g.os, n, lo, hi);
  else window(s, g.kw, g.os, n, lo, hi);
}
template <typename T>
inline T tapw(const Geom<T>& g, T s, int c) {
  if (g.float_taps)
    return (T)lut_weight<float>((float)s, c, (float)g.os, (float)g.kw, g.lut32.data(), g.lut32.size());
  return lut_weight(s, c, g.os, g.kw, g.lut.data(), g.lut.size());
}

// Forward interpolation: y_i = sum over the window of w * grid[ny + nx*Gy (+ nz*Gx*Gy)]
// (gridding.cpp:217-415).
template <typename T>
void interp_forward(const Geom<T>& g, u64 M, const T* kx, const T* ky, const T* kz,
                    const std::complex<T>* grid, std::complex<T>* y) {
  for (u64 i = 0; i < M; ++i) {
    T acc_r = 0, acc_i = 0;
    T sx = grid_pos(g, kx[i], g.Nx);
    T sy = grid_pos(g, ky[i], g.Ny);
    int xl, xh, yl, yh;
    win(g, sx, g.Nx, xl, xh);
    win(g, sy, g.Ny, yl, yh);
    if (!g.is3d()) {
      for (int nx = xl; nx <= xh; ++nx) {
        T wx = tapw(g, sx, nx);
        for (int ny = yl; ny <= yh; ++ny) {
          T wy = tapw(g, sy, ny);
          T w = wx * wy;
          const std::complex<T> v = grid[(u64)ny + (u64)nx * g.Gy];
          acc_r += w * v.real();
          acc_i += w * v.imag();
        }
      }
    } else {
      T sz = grid_pos(g, kz[i], g.Nz);
      int zl, zh;
      win(g, sz, g.Nz, zl, zh);
      for (int nz = zl; nz <= zh; ++nz) {
        T wz = tapw(g, sz, nz);
        for (int nx = xl; nx <= xh; ++nx) {
          T wx = tapw(g, sx, nx);
          for (int ny = yl; ny <= yh; ++ny) {
            T wy = tapw(g, sy, ny);
            T w = wx * wy * wz;
            const std::complex<T> v = grid[(u64)ny + (u64)nx * g.Gy + (u64)nz * g.Gx * g.Gy];
            acc_r += w * v.real();
            acc_i += w * v.imag();
          }
        }
      }
    }
    y[i] = std::complex<T>(acc_r, acc_i);
  }
}

// Adjoint spreading in sample order: grid[idx] += w * d_i (gridding.cpp:31-214).
template <typename T>
void spread_adjoint(const Geom<T>& g, u64 M, const T* kx, const T* ky, const T* kz,
                    const std::complex<T>* d, std::complex<T>* grid) {
  T* gr = reinterpret_cast<T*>(grid);
  for (u64 i = 0; i < M; ++i) {
    const T dr = d[i].real(), di = d[i].imag();
    T sx = grid_pos(g, kx[i], g.Nx);
    T sy = grid_pos(g, ky[i], g.Ny);
    int xl, xh, yl, yh;
    win(g, sx, g.Nx, xl, xh);
    win(g, sy, g.Ny, yl, yh);
    if (!g.is3d()) {
      for (int nx = xl; nx <= xh; ++nx) {
        T wx = tapw(g, sx, nx);
        for (int ny = yl; ny <= yh; ++ny) {
          T wy = tapw(g, sy, ny);
          T w = wx * wy;
          const u64 idx = 2 * ((u64)ny + (u64)nx * g.Gy);
          gr[idx] += w * dr;
          gr[idx + 1] += w * di;
        }
      }
    } else {
      T sz = grid_pos(g, kz[i], g.Nz);
      int zl, zh;
      win(g, sz, g.Nz, zl, zh);
      for (int nz = zl; nz <= zh; ++nz) {
        T wz = tapw(g, sz, nz);
        for (int nx = xl; nx <= xh; ++nx) {
          T wx = tapw(g, sx, nx);
          for (int ny = yl; ny <= yh; ++ny) {
            T wy = tapw(g, sy, ny);
            T w = wx * wy * wz;
            const u64 idx = (u64)ny + (u64)nx * g.Gy + (u64)nz * g.Gx * g.Gy;
            gr[2 * idx] += w * dr;
            gr[2 * idx + 1] += w * di;
          }
        }
      }
    }
  }
}

// Reciprocal Kaiser-Bessel transform factor along one axis
// (griddingSupport.cpp:249-260 in 2-D; :331-348 in 3-D, where the sinh branch
// runs in double).
template <typename T>
inline T deapod_axis(T u, T kw, T beta, bool three_d) {
  T c = (T)(kPiF * kPiF) * kw * kw * u * u - beta * beta;
  if (c >= 0) return (T)(std::sin(std::sqrt(c)) / std::sqrt(c));
  if (three_d) return (T)(std::sinh(std::sqrt(-1.0 * c)) / std::sqrt(-1.0 * c));
  return std::sinh(std::sqrt((T)-1.0 * c)) / std::sqrt((T)-1.0 * c);
}

// deapodization2d/3d: out = in / Pi_axes g(u) / os^d; NaN factor -> 0
// (griddingSupport.cpp:210-368).  In place on an image (y fastest).
template <typename T>
void deapodize(const Geom<T>& g, std::complex<T>* img) {
  const int X = g.Nx, Y = g.Ny, Z = g.Nz;
  if (!g.is3d()) {
    for (int x = 0; x < X; ++x) {
      for (int y = 0; y < Y; ++y) {
        T uy = (T)(y - (Y / 2)) / (T)Y;
        T ux = (T)(x - (X / 2)) / (T)X;
        T k = deapod_axis(ux, g.kw, g.beta, false) * deapod_axis(uy, g.kw, g.beta, false);
        const u64 p = (u64)y + (u64)x * Y;
        if (k == k) {
          T os2 = g.os * g.os;
          img[p] = std::complex<T>(img[p].real() / k * ((T)1.0 / os2), img[p].imag() / k * ((T)1.0 / os2));
        } else {
          img[p] = std::complex<T>(0, 0);
        }
      }
    }
  } else {
    for (int z = 0; z < Z; ++z)
      for (int x = 0; x < X; ++x)
        for (int y = 0; y < Y; ++y) {
          T uz = (T)((z) - ((T)Z / 2.0)) / (T)Z;
          T uy = (T)((y) - ((T)Y / 2.0)) / (T)Y;
          T ux = (T)((x) - ((T)X / 2.0)) / (T)X;
          T kx = deapod_axis(ux, g.kw, g.beta, true);
          T ky = deapod_axis(uy, g.kw, g.beta, true);
          T kz = deapod_axis(uz, g.kw, g.beta, true);
          T k = kx * ky * kz;
          const u64 p = (u64)z * Y * X + (u64)x * Y + y;
          if (k == k) {
            T os3 = g.os * g.os * g.os;
            img[p] = std::complex<T>((T)((img[p].real()) / k * (1.0 / os3)),
                                     (T)((img[p].imag()) / k * (1.0 / os3)));
          } else {
            img[p] = std::complex<T>(0, 0);
          }
        }
  }
}

// Circular shift by (sa, sb, sc) of an array with a fastest (extent na)
// (griddingSupport.cpp:552-593): out[(a+sa)%na, (b+sb)%nb, (c+sc)%nc] = in[a,b,c].
template <typename T>
void circshift(std::complex<T>* out, const std::complex<T>* in, int na, int nb, int nc, int sa, int sb, int sc) {
  for (int c = 0; c < nc; ++c)
    for (int b = 0; b < nb; ++b)
      for (int a = 0; a < na; ++a) {
        const u64 src = (u64)a + (u64)b * na + (u64)c * na * nb;
        const u64 dst = (u64)((a + sa) % na) + (u64)((b + sb) % nb) * na + (u64)((c + sc) % nc) * na * nb;
        out[dst] = in[src];
      }
}

// fftshift: floor(n/2) per axis; ifftshift: ceil(n/2) in-plane, floor(n/2)
// along z (griddingSupport.cpp:599-627).  Axes passed as (xdim, ydim, zdim) =
// gridSize[0..2], with xdim the fastest index, as the reference does.
template <typename T>
void fftshift_grid(const Geom<T>& g, std::complex<T>* out, const std::complex<T>* in) {
  circshift(out, in, g.Gx, g.Gy, g.Gz, (int)std::floor(g.Gx / 2.0), (int)std::floor(g.Gy / 2.0),
            g.is3d() ? (int)std::floor(g.Gz / 2.0) : 0);
}
template <typename T>
void ifftshift_grid(const Geom<T>& g, std::complex<T>* out, const std::complex<T>* in) {
  circshift(out, in, g.Gx, g.Gy, g.Gz, (int)std::ceil(g.Gx / 2.0), (int)std::ceil(g.Gy / 2.0),
            g.is3d() ? (int)std::floor(g.Gz / 2.0) : 0);
}

// zero_pad2d/3d (griddingSupport.cpp:457-547) and crop_center_region2d/3d
// (griddingSupport.cpp:372-453): centre embed / extract.
template <typename T>
void zero_pad(const Geom<T>& g, std::complex<T>* grid, const std::complex<T>* img) {
  std::fill(grid, grid + g.ngrid(), std::complex<T>(0, 0));
  if (!g.is3d()) {
    // zero_pad2d indexes the first image axis fastest (griddingSupport.cpp:488-489).
    const int oy = (int)(((T)g.Ny * g.os / (T)2.0) - ((T)g.Ny / (T)2.0));
    const int ox = (int)(((T)g.Nx * g.os / (T)2.0) - ((T)g.Nx / (T)2.0));
    const int rowlen = (int)(g.Nx * g.os);
    for (int b = 0; b < g.Ny; ++b)
      for (int a = 0; a < g.Nx; ++a)
        grid[(u64)(b + oy) * rowlen + (a + ox)] = img[(u64)b * g.Nx + a];
  } else {
    const int oy = (int)(((T)g.Ny * g.os / (T)2.0) - ((T)g.Ny / (T)2.0));
    const int ox = (int)(((T)g.Nx * g.os / (T)2.0) - ((T)g.Nx / (T)2.0));
    const int oz = (int)(((T)g.Nz * g.os / (T)2.0) - ((T)g.Nz / (T)2.0));
    for (int z = 0; z < g.Nz; ++z)
      for (int y = 0; y < g.Ny; ++y)
        for (int x = 0; x < g.Nx; ++x) {
          const u64 dst = (u64)(int)((z + oz) * g.Nx * g.Ny * g.os * g.os) + (u64)(x + ox) * (int)(g.Ny * g.os) + (y + oy);
          grid[dst] = img[(u64)z * g.Nx * g.Ny + (u64)x * g.Ny + y];
        }
  }
}
template <typename T>
void crop_center(const Geom<T>& g, std::complex<T>* img, const std::complex<T>* grid) {
  const int oy = (int)(((T)g.Gy / (T)2.0) - ((T)g.Ny / (T)2.0));
  const int ox = (int)(((T)g.Gx / (T)2.0) - ((T)g.Nx / (T)2.0));
  const int oz = g.is3d() ? (int)(((T)g.Gz / (T)2.0) - ((T)g.Nz / (T)2.0)) : 0;
  for (int z = 0; z < g.Nz; ++z)
    for (int x = 0; x < g.Nx; ++x)
      for (int y = 0; y < g.Ny; ++y)
        img[(u64)z * g.Nx * g.Ny + (u64)x * g.Ny + y] =
            grid[(u64)(z + oz) * g.Gx * g.Gy + (u64)(x + ox) * g.Gy + (y + oy)];
}

// In-place unnormalised FFT over the grid with the dimension order fftCPU.cpp
// gives FFTW: plan_dft_2d(Gy, Gx), plan_dft_3d(Gz, Gy, Gx) (fftCPU.cpp:54, 84).
template <typename T>
void grid_fft(const Geom<T>& g, std::complex<T>* grid, int sign) {
  if (!g.is3d()) {
    const std::size_t dims[2] = {(std::size_t)g.Gy, (std::size_t)g.Gx};
    fft_nd<T>(grid, dims, 2, sign);
  } else {
    const std::size_t dims[3] = {(std::size_t)g.Gz, (std::size_t)g.Gy, (std::size_t)g.Gx};
    fft_nd<T>(grid, dims, 3, sign);
  }
}

// ---------------------------------------------------------------------------
// Backend hook: the composites below run either on the restated kernels or
// on the reference's own compiled kernels (oracle/_ref/libpgref.so).
// ---------------------------------------------------------------------------
template <typename T>
struct RefKernels {
  // computeFd_CPU_Grid / computeFH_CPU_Grid wrappers
  void (*fd)(int, const T*, const T*, const T*, const T*, int, int, int, T, T, T, const T*, u64, T*) = nullptr;
  void (*fh)(int, const T*, const T*, const T*, const T*, int, int, int, T, T, T, const T*, u64, T*) = nullptr;
  // ftCpu / iftCpu wrappers
  void (*ft)(T*, T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*,
             const T*, const T*, int, int) = nullptr;
  void (*ift)(T*, T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*,
              const T*, const T*, int, int) = nullptr;
  // ftCpuWithGrads / iftCpuWithGrads wrappers
  void (*ftg)(T*, T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*,
              const T*, const T*, const T*, const T*, int, int, int, int, int) = nullptr;
  void (*iftg)(T*, T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*, const T*,
               const T*, const T*, const T*, const T*, int, int, int, int, int) = nullptr;
  // forwardSpatialInterp / adjointSpatialInterp bodies
  void (*ifwd)(int, const T*, const T*, const T*, const T*, u64, int, int, int, T, T, T, const T*, u64, T*) = nullptr;
  void (*iadj)(int, const T*, const T*, const T*, const T*, u64, int, int, int, T, T, T, const T*, u64, T*) = nullptr;
};
template <typename T>
RefKernels<T>& ref_kernels() {
  static RefKernels<T> k;
  return k;
}

// ---------------------------------------------------------------------------
// Operators.  n1 = data length, n2 = image length (reference naming).
// ---------------------------------------------------------------------------
template <typename T>
struct Op {
  using C = std::complex<T>;
  u64 n1 = 0, n2 = 0;
  virtual ~Op() {}
  virtual void forward(const C* x, C* y) const = 0;   // operator*
  virtual void adjoint(const C* y, C* x) const = 0;   // operator/
};

// Gnufft (Gnufft.cpp:34-211).
template <typename T>
struct GnufftOp : Op<T> {
  using C = std::complex<T>;
  Geom<T> g;
  std::vector<T> kx, ky, kz;
  bool use_ref = false;

  GnufftOp(u64 M, T gridos, int nx, int ny, int nz, const T* k1, const T* k2, const T* k3) {
    this->n1 = (u64)nx * ny * nz;   // image (Gnufft names the image n1)
    this->n2 = M;                   // samples
    g = Geom<T>::make(nx, ny, nz, gridos);
    kx.assign(k1, k1 + M); ky.assign(k2, k2 + M); kz.assign(k3, k3 + M);
  }
  u64 data_len() const { return this->n2; }
  u64 image_len() const { return this->n1; }
  // Evaluate the float operator's taps in this (double) instantiation.
  void use_float_taps() {
    const float beta32 = kb_beta<float>((float)g.os, 4.0f);
    g.float_taps = true;
    g.lut32 = kb_lut<float>(beta32, 4.0f);
    g.beta = (T)beta32;   // the float operator's beta (deapodization), widened
  }

  // computeFd_CPU_Grid restated (gridding.cpp:584-727)
  void forward(const C* x, C* y) const override {
    const u64 M = this->n2;
    if (use_ref && ref_kernels<T>().fd) {
      ref_kernels<T>().fd((int)M, kx.data(), ky.data(), kz.data(), reinterpret_cast<const T*>(x), g.Nx, g.Ny,
                          g.Nz, g.os, g.kw, g.beta, g.lut.data(), g.lut.size(), reinterpret_cast<T*>(y));
      return;
    }
    std::vector<C> img(x, x + g.nimg());
    deapodize(g, img.data());
    std::vector<C> a(g.ngrid()), b(g.ngrid());
    zero_pad(g, a.data(), img.data());
    fftshift_grid(g, b.data(), a.data());
    grid_fft(g, b.data(), -1);
    ifftshift_grid(g, a.data(), b.data());
    interp_forward(g, M, kx.data(), ky.data(), kz.data(), a.data(), y);
  }
  // computeFH_CPU_Grid restated (gridding.cpp:418-581)
  void adjoint(const C* d, C* x) const override {
    const u64 M = this->n2;
    if (use_ref && ref_kernels<T>().fh) {
      ref_kernels<T>().fh((int)M, kx.data(), ky.data(), kz.data(), reinterpret_cast<const T*>(d), g.Nx, g.Ny,
                          g.Nz, g.os, g.kw, g.beta, g.lut.data(), g.lut.size(), reinterpret_cast<T*>(x));
      return;
    }
    std::vector<C> a(g.ngrid(), C(0, 0)), b(g.ngrid());
    spread_adjoint(g, M, kx.data(), ky.data(), kz.data(), d, a.data());
    ifftshift_grid(g, b.data(), a.data());
    grid_fft(g, b.data(), +1);
    fftshift_grid(g, a.data(), b.data());
    crop_center(g, x, a.data());
    deapodize(g, x);
  }
  // Gnufft::forwardSpatialInterp (Gnufft.cpp:213-258): grid -> samples, no FFT
  void forward_interp(const C* grid, C* y) const {
    const u64 M = this->n2;
    if (use_ref && ref_kernels<T>().ifwd) {
      ref_kernels<T>().ifwd((int)M, kx.data(), ky.data(), kz.data(), reinterpret_cast<const T*>(grid), g.ngrid(),
                            g.Nx, g.Ny, g.Nz, g.os, g.kw, g.beta, g.lut.data(), g.lut.size(), reinterpret_cast<T*>(y));
      return;
    }
    interp_forward(g, M, kx.data(), ky.data(), kz.data(), grid, y);
  }
  // Gnufft::adjointSpatialInterp (Gnufft.cpp:261-330): samples -> zeroed grid + spread
  void adjoint_interp(const C* d, C* grid) const {
    const u64 M = this->n2;
    if (use_ref && ref_kernels<T>().iadj) {
      ref_kernels<T>().iadj((int)M, kx.data(), ky.data(), kz.data(), reinterpret_cast<const T*>(d), g.ngrid(), g.Nx,
                            g.Ny, g.Nz, g.os, g.kw, g.beta, g.lut.data(), g.lut.size(), reinterpret_cast<T*>(grid));
      return;
    }
    std::fill(grid, grid + g.ngrid(), C(0, 0));
    spread_adjoint(g, M, kx.data(), ky.data(), kz.data(), d, grid);
  }
};

// calc3DDensityCompensation (reconSupport/directRecon.cpp:28-61).  Armadillo
// divides a complex column by a real one or by a scalar after promoting the
// divisor to complex, so the divisions here are complex / complex.
template <typename T>
std::vector<T> density_compensation(const T* kx, const T* ky, const T* kz, u64 n, int ninplane, int nz,
                                    bool use_ref) {
  using C = std::complex<T>;
  GnufftOp<T> G(n, (T)3.0, ninplane, ninplane, nz, kx, ky, kz);  // overSampling = 3 (:32-35)
  G.use_ref = use_ref;
  std::vector<C> dcf(n, C(1, 0));
  const C den((T)n * (T)n);
  for (auto& v : dcf) v /= den;                                  // :38-40
  std::vector<C> c1(G.g.ngrid()), c2(n);
  for (int it = 0; it < 2; ++it) {                               // Niter = 2 (:30), :49-55
    G.adjoint_interp(dcf.data(), c1.data());
    G.forward_interp(c1.data(), c2.data());
    for (u64 i = 0; i < n; ++i) dcf[i] = dcf[i] / C(c2[i].real());
  }
  // normalise(dcf, 2) (:57): Armadillo's 2-norm of a complex column sums
  // |v|^2 and, if that underflows or overflows, rescales by the largest |v|
  T acc = 0;
  for (const auto& v : dcf) {
    const T a = std::abs(v);
    acc += a * a;
  }
  T nrm = std::sqrt(acc);
  if (nrm == (T)0 || !std::isfinite(nrm)) {
    T mx = 0;
    for (const auto& v : dcf) mx = std::max(mx, std::abs(v));
    T alt = 0;
    if (mx > (T)0 && std::isfinite(mx))
      for (const auto& v : dcf) {
        const T a = std::abs(v) / mx;
        alt += a * a;
      }
    nrm = (mx > (T)0 && std::isfinite(mx)) ? std::sqrt(alt) * mx : nrm;
  }
  std::vector<T> out(n);
  for (u64 i = 0; i < n; ++i) out[i] = std::abs(nrm != (T)0 ? dcf[i] / C(nrm) : dcf[i]);  // abs (:59)
  return out;
}

// Gdft (Gdft.cpp:33-136).  exact64 selects the FP64 oracle formula (double
// sin/cos); otherwise the expression types of ftCpu / iftCpu are kept
// (float sinf/cosf, ftCpu.cpp:104, 129-130, 203-204).
template <typename T>
struct GdftOp : Op<T> {
  using C = std::complex<T>;
  std::vector<T> kx, ky, kz, ix, iy, iz, fm, t;
  bool exact64 = false;
  bool use_ref = false;
  GdftOp(u64 nk, u64 ni, const T* k1, const T* k2, const T* k3, const T* i1, const T* i2, const T* i3,
         const T* f, const T* tt) {
    this->n1 = nk; this->n2 = ni;
    kx.assign(k1, k1 + nk); ky.assign(k2, k2 + nk); kz.assign(k3, k3 + nk);
    ix.assign(i1, i1 + ni); iy.assign(i2, i2 + ni); iz.assign(i3, i3 + ni);
    fm.assign(f, f + ni); t.assign(tt, tt + nk);
  }
  void forward(const C* x, C* y) const override {
    const u64 nk = this->n1, ni = this->n2;
    std::vector<T> xr(ni), xi(ni), yr(nk, 0), yi(nk, 0);
    for (u64 j = 0; j < ni; ++j) { xr[j] = x[j].real(); xi[j] = x[j].imag(); }
    if (use_ref && ref_kernels<T>().ft && !exact64) {
      ref_kernels<T>().ft(yr.data(), yi.data(), xr.data(), xi.data(), kx.data(), ky.data(), kz.data(), ix.data(),
                          iy.data(), iz.data(), fm.data(), t.data(), (int)nk, (int)ni);
    } else if (exact64) {
      const double tpi = 2.0 * kPiD;
      for (u64 i = 0; i < nk; ++i) {
        double sr = 0, si = 0;
        for (u64 j = 0; j < ni; ++j) {
          double ph = tpi * ((double)kx[i] * ix[j] + (double)ky[i] * iy[j] + (double)kz[i] * iz[j]) +
                      (double)fm[j] * t[i];
          double s = std::sin(ph), c = std::cos(ph);
          sr += c * xr[j] + s * xi[j];
          si += -s * xr[j] + c * xi[j];
        }
        yr[i] = (T)sr; yi[i] = (T)si;
      }
    } else {
      // ftCpu.cpp:115-138
      for (u64 i = 0; i < nk; ++i) {
        T sr = 0.0, si = 0.0;
        T a = kx[i] * 2 * kPiF, b = ky[i] * 2 * kPiF, c = kz[i] * 2 * kPiF;
        T ti = t[i];
        for (u64 j = 0; j < ni; ++j) {
          T e = (a * ix[j] + b * iy[j] + c * iz[j] + (fm[j] * ti));
          float s = sinf(e);
          float co = cosf(e);
          sr += (co * xr[j]) + (s * xi[j]);
          si += (-s * xr[j]) + (co * xi[j]);
        }
        yr[i] = sr; yi[i] = si;
      }
    }
    for (u64 i = 0; i < nk; ++i) y[i] = C(yr[i], yi[i]);
  }
  void adjoint(const C* y, C* x) const override {
    const u64 nk = this->n1, ni = this->n2;
    std::vector<T> yr(nk), yi(nk), xr(ni, 0), xi(ni, 0);
    for (u64 i = 0; i < nk; ++i) { yr[i] = y[i].real(); yi[i] = y[i].imag(); }
    if (use_ref && ref_kernels<T>().ift && !exact64) {
      ref_kernels<T>().ift(xr.data(), xi.data(), yr.data(), yi.data(), kx.data(), ky.data(), kz.data(), ix.data(),
                           iy.data(), iz.data(), fm.data(), t.data(), (int)nk, (int)ni);
    } else if (exact64) {
      const double tpi = 2.0 * kPiD;
      for (u64 j = 0; j < ni; ++j) {
        double sr = 0, si = 0;
        for (u64 i = 0; i < nk; ++i) {
          double ph = tpi * ((double)kx[i] * ix[j] + (double)ky[i] * iy[j] + (double)kz[i] * iz[j]) +
                      (double)fm[j] * t[i];
          double s = std::sin(ph), c = std::cos(ph);
          sr += c * yr[i] - s * yi[i];
          si += s * yr[i] + c * yi[i];
        }
        xr[j] = (T)sr; xi[j] = (T)si;
      }
    } else {
      // iftCpu.cpp:164-212
      T tpi = kPiF * 2.0;
      for (u64 j = 0; j < ni; ++j) {
        T sr = 0.0, si = 0.0;
        T ax = ix[j] * tpi, ay = iy[j] * tpi, az = iz[j] * tpi;
        T f = fm[j];
        for (u64 i = 0; i < nk; ++i) {
          T e = (kx[i] * ax + ky[i] * ay + kz[i] * az + (f * t[i]));
          T s = sinf(e);
          T co = cosf(e);
          sr += (co * yr[i]) - (s * yi[i]);
          si += (s * yr[i]) + (co * yi[i]);
        }
        xr[j] = sr; xi[j] = si;
      }
    }
    for (u64 j = 0; j < ni; ++j) x[j] = C(xr[j], xi[j]);
  }
};

// GdftR2 (GdftR2.cpp:32-150): Gdft with per-pair through-voxel dephasing
// factors from the field map's differences (ftCpuWithGrads.cpp:76-216).
template <typename T>
struct GdftR2Op : GdftOp<T> {
  using C = std::complex<T>;
  std::vector<T> gx, gy, gz;
  int nx, ny, nz;
  // sincPG (ftCpuWithGrads.cpp:76-84): the product with the float MRI_PI and
  // sin in T (the overload for T; checked bit for bit against the compiled
  // reference)
  static T sinc_pg(T x) {
    if (std::fabs((double)x) < 0.0001) return (T)1.0;
    return (T)(std::sin(kPiF * x) / (kPiF * x));
  }
  static double sinc64(double x) { return std::fabs(x) < 0.0001 ? 1.0 : std::sin(kPiD * x) / (kPiD * x); }
  // Cd of GdftR2.cpp:72-110
  std::vector<T> cd(u64 off) const {
    const u64 N = (u64)nx * ny * nz;
    std::vector<T> out(N, (T)0);
    for (u64 ii = off; ii < N - off; ++ii) out[ii] = this->fm[ii + off] - this->fm[ii - off];
    for (u64 ii = 0; ii < off; ++ii) out[ii] = this->fm[ii + off] - this->fm[ii];
    for (u64 ii = N - off; ii < N; ++ii) out[ii] = this->fm[ii] - this->fm[ii - off];
    return out;
  }
  GdftR2Op(u64 nk, u64 ni, const T* k1, const T* k2, const T* k3, const T* i1, const T* i2, const T* i3, const T* f,
           const T* tt, int x, int y, int z)
      : GdftOp<T>(nk, ni, k1, k2, k3, i1, i2, i3, f, tt), nx(x), ny(y), nz(z) {
    gx = cd(1);
    gy = cd((u64)ny);
    gz = cd((u64)nx * ny);
  }
  void forward(const C* xin, C* y) const override {
    const u64 nk = this->n1, ni = this->n2;
    std::vector<T> xr(ni), xi(ni), yr(nk, 0), yi(nk, 0);
    for (u64 j = 0; j < ni; ++j) { xr[j] = xin[j].real(); xi[j] = xin[j].imag(); }
    const auto& kx = this->kx; const auto& ky = this->ky; const auto& kz = this->kz;
    const auto& ix = this->ix; const auto& iy = this->iy; const auto& iz = this->iz;
    const auto& fm = this->fm; const auto& t = this->t;
    if (this->use_ref && ref_kernels<T>().ftg && !this->exact64) {
      ref_kernels<T>().ftg(yr.data(), yi.data(), xr.data(), xi.data(), kx.data(), ky.data(), kz.data(), ix.data(),
                           iy.data(), iz.data(), fm.data(), gx.data(), gy.data(), gz.data(), t.data(), (int)nk,
                           (int)ni, nx, ny, nz);
    } else if (this->exact64) {
      const double tpi = 2.0 * kPiD;
      for (u64 i = 0; i < nk; ++i) {
        double sr = 0, si = 0;
        for (u64 j = 0; j < ni; ++j) {
          const double ph = tpi * ((double)kx[i] * ix[j] + (double)ky[i] * iy[j] + (double)kz[i] * iz[j]) +
                            (double)fm[j] * t[i];
          const double b = sinc64((double)kx[i] / nx + (double)gx[j] * t[i]) *
                           sinc64((double)ky[i] / ny + (double)gy[j] * t[i]) *
                           sinc64((double)kz[i] / nz + (double)gz[j] * t[i]);
          const double s = std::sin(ph), c = std::cos(ph);
          sr += b * (c * xr[j] + s * xi[j]);
          si += b * (-s * xr[j] + c * xi[j]);
        }
        yr[i] = (T)sr; yi[i] = (T)si;
      }
    } else {
      // ftCpuWithGrads.cpp:115-138
      for (u64 i = 0; i < nk; ++i) {
        T sr = 0.0, si = 0.0;
        T a = kx[i] * 2 * kPiF, b = ky[i] * 2 * kPiF, c = kz[i] * 2 * kPiF;
        T ti = t[i];
        for (u64 j = 0; j < ni; ++j) {
          T e = (a * ix[j] + b * iy[j] + c * iz[j] + (fm[j] * ti));
          float s = sinf(e);
          float co = cosf(e);
          T bf = sinc_pg(kx[i] / nx + gx[j] * ti) * sinc_pg(ky[i] / ny + gy[j] * ti) * sinc_pg(kz[i] / nz + gz[j] * ti);
          sr += bf * ((co * xr[j]) + (s * xi[j]));
          si += bf * ((-s * xr[j]) + (co * xi[j]));
        }
        yr[i] = sr; yi[i] = si;
      }
    }
    for (u64 i = 0; i < nk; ++i) y[i] = C(yr[i], yi[i]);
  }
  void adjoint(const C* yin, C* x) const override {
    const u64 nk = this->n1, ni = this->n2;
    std::vector<T> yr(nk), yi(nk), xr(ni, 0), xi(ni, 0);
    for (u64 i = 0; i < nk; ++i) { yr[i] = yin[i].real(); yi[i] = yin[i].imag(); }
    const auto& kx = this->kx; const auto& ky = this->ky; const auto& kz = this->kz;
    const auto& ix = this->ix; const auto& iy = this->iy; const auto& iz = this->iz;
    const auto& fm = this->fm; const auto& t = this->t;
    if (this->use_ref && ref_kernels<T>().iftg && !this->exact64) {
      ref_kernels<T>().iftg(xr.data(), xi.data(), yr.data(), yi.data(), kx.data(), ky.data(), kz.data(), ix.data(),
                            iy.data(), iz.data(), fm.data(), gx.data(), gy.data(), gz.data(), t.data(), (int)nk,
                            (int)ni, nx, ny, nz);
    } else if (this->exact64) {
      const double tpi = 2.0 * kPiD;
      for (u64 j = 0; j < ni; ++j) {
        double sr = 0, si = 0;
        for (u64 i = 0; i < nk; ++i) {
          const double ph = tpi * ((double)kx[i] * ix[j] + (double)ky[i] * iy[j] + (double)kz[i] * iz[j]) +
                            (double)fm[j] * t[i];
          const double b = sinc64((double)kx[i] / nx + (double)gx[j] * t[i]) *
                           sinc64((double)ky[i] / ny + (double)gy[j] * t[i]) *
                           sinc64((double)kz[i] / nz + (double)gz[j] * t[i]);
          const double s = std::sin(ph), c = std::cos(ph);
          sr += b * (c * yr[i] - s * yi[i]);
          si += b * (s * yr[i] + c * yi[i]);
        }
        xr[j] = (T)sr; xi[j] = (T)si;
      }
    } else {
      // ftCpuWithGrads.cpp:164-212
      T tpi = kPiF * 2.0;
      for (u64 j = 0; j < ni; ++j) {
        T sr = 0.0, si = 0.0;
        T ax = ix[j] * tpi, ay = iy[j] * tpi, az = iz[j] * tpi;
        T f = fm[j];
        for (u64 i = 0; i < nk; ++i) {
          T e = (kx[i] * ax + ky[i] * ay + kz[i] * az + (f * t[i]));
          T s = sinf(e);
          T co = cosf(e);
          T bf = sinc_pg(kx[i] / nx + gx[j] * t[i]) * sinc_pg(ky[i] / ny + gy[j] * t[i]) *
                 sinc_pg(kz[i] / nz + gz[j] * t[i]);
          sr += bf * ((co * yr[i]) - (s * yi[i]));
          si += bf * ((s * yr[i]) + (co * yi[i]));
        }
        xr[j] = sr; xi[j] = si;
      }
    }
    for (u64 j = 0; j < ni; ++j) x[j] = C(xr[j], xi[j]);
  }
};

template <typename T>
struct SenseOp;

// Data/image lengths of any operator: Gnufft names the image n1
// (Gnufft.cpp:42-43) and SENSE's n1 is the per-coil data length
// (SENSE.cpp:36, 42), so both need a translation.
template <typename T>
inline u64 op_data_len(const Op<T>& op);
template <typename T>
inline u64 op_image_len(const Op<T>& op) {
  if (auto* g = dynamic_cast<const GnufftOp<T>*>(&op)) return g->image_len();
  return op.n2;
}

// ---------------------------------------------------------------------------
// Dense complex algebra in the operator's precision for the min-max
// interpolators (Armadillo inv / pinv / cond / rcond over LAPACK in the
// reference; restated: Gauss-Jordan with partial pivoting, one-sided Jacobi
// SVD, pseudo-inverse with Armadillo's default tolerance n * max(s) * eps,
// and the 1-norm reciprocal condition number that LAPACK's gecon estimates).
// ---------------------------------------------------------------------------
template <typename T>
using CM = std::vector<std::complex<T>>;  // n x n row-major

template <typename T>
bool la_inverse(CM<T> A, int n, CM<T>* out) {
  using C = std::complex<T>;
  CM<T> I((size_t)n * n, C(0, 0));
  for (int i = 0; i < n; ++i) I[(size_t)i * n + i] = C(1, 0);
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::abs(A[(size_t)r * n + c]) > std::abs(A[(size_t)p * n + c])) p = r;
    if (A[(size_t)p * n + c] == C(0, 0)) return false;
    if (p != c)
      for (int k = 0; k < n; ++k) {
        std::swap(A[(size_t)p * n + k], A[(size_t)c * n + k]);
        std::swap(I[(size_t)p * n + k], I[(size_t)c * n + k]);
      }
    const C inv = C(1, 0) / A[(size_t)c * n + c];
    for (int k = 0; k < n; ++k) {
      A[(size_t)c * n + k] *= inv;
      I[(size_t)c * n + k] *= inv;
    }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const C f = A[(size_t)r * n + c];
      if (f == C(0, 0)) continue;
      for (int k = 0; k < n; ++k) {
        A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
        I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
      }
    }
  }
  *out = I;
  return true;
}

// A = U diag(s) V^H by one-sided (Hestenes) Jacobi rotations.
template <typename T>
void la_svd(const CM<T>& A, int n, std::vector<T>* s, CM<T>* U, CM<T>* V) {
  using C = std::complex<T>;
  CM<T> W = A, Vm((size_t)n * n, C(0, 0));
  for (int i = 0; i < n; ++i) Vm[(size_t)i * n + i] = C(1, 0);
  const T tol = std::numeric_limits<T>::epsilon();
  for (int sweep = 0; sweep < 60; ++sweep) {
    T off = 0;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        T app = 0, aqq = 0;
        C apq(0, 0);
        for (int i = 0; i < n; ++i) {
          app += std::norm(W[(size_t)i * n + p]);
          aqq += std::norm(W[(size_t)i * n + q]);
          apq += std::conj(W[(size_t)i * n + p]) * W[(size_t)i * n + q];
        }
        const T mag = std::abs(apq);
        if (mag == (T)0 || mag <= tol * std::sqrt(app * aqq)) continue;
        off = std::max(off, mag / std::sqrt(app * aqq));
        const C ph = apq / mag;
        const T zeta = (aqq - app) / ((T)2 * mag);
        const T t = (zeta >= 0 ? (T)1 : (T)-1) / (std::abs(zeta) + std::sqrt((T)1 + zeta * zeta));
        const T c = (T)1 / std::sqrt((T)1 + t * t), sn = c * t;
        for (int i = 0; i < n; ++i) {
          const C wp = W[(size_t)i * n + p], wq = W[(size_t)i * n + q];
          W[(size_t)i * n + p] = c * wp - sn * std::conj(ph) * wq;
          W[(size_t)i * n + q] = sn * ph * wp + c * wq;
          const C vp = Vm[(size_t)i * n + p], vq = Vm[(size_t)i * n + q];
          Vm[(size_t)i * n + p] = c * vp - sn * std::conj(ph) * vq;
          Vm[(size_t)i * n + q] = sn * ph * vp + c * vq;
        }
      }
    if (off < tol) break;
  }
  s->assign(n, (T)0);
  CM<T> Um((size_t)n * n, C(0, 0));
  for (int j = 0; j < n; ++j) {
    T nr = 0;
    for (int i = 0; i < n; ++i) nr += std::norm(W[(size_t)i * n + j]);
    nr = std::sqrt(nr);
    (*s)[j] = nr;
    for (int i = 0; i < n; ++i) Um[(size_t)i * n + j] = nr > 0 ? W[(size_t)i * n + j] / nr : C(0, 0);
  }
  *U = Um;
  *V = Vm;
}

template <typename T>
CM<T> la_pinv(const CM<T>& A, int n) {
  std::vector<T> s;
  CM<T> U, V;
  la_svd(A, n, &s, &U, &V);
  const T smax = *std::max_element(s.begin(), s.end());
  const T tol = (T)n * smax * std::numeric_limits<T>::epsilon();
  CM<T> P((size_t)n * n, std::complex<T>(0, 0));
  for (int k = 0; k < n; ++k) {
    if (s[k] <= tol) continue;
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c)
        P[(size_t)r * n + c] += V[(size_t)r * n + k] * ((T)1 / s[k]) * std::conj(U[(size_t)c * n + k]);
  }
  return P;
}

template <typename T>
T la_cond(const CM<T>& A, int n) {
  std::vector<T> s;
  CM<T> U, V;
  la_svd(A, n, &s, &U, &V);
  const T smin = *std::min_element(s.begin(), s.end());
  return smin > 0 ? *std::max_element(s.begin(), s.end()) / smin : std::numeric_limits<T>::infinity();
}

template <typename T>
T la_norm1(const CM<T>& A, int n) {
  T m = 0;
  for (int c = 0; c < n; ++c) {
    T sum = 0;
    for (int r = 0; r < n; ++r) sum += std::abs(A[(size_t)r * n + c]);
    m = std::max(m, sum);
  }
  return m;
}

// Min-max interpolator (TimeSegmentation.cpp:94-156) for one shot: AA(m, l),
// m < none, l < L, column-major like tempAA.
template <typename T>
std::vector<std::complex<T>> aa_minmax(const T* fm, u64 n2, const std::vector<T>& tv, u64 none, int L, T tau) {
  using C = std::complex<T>;
  const C I(0, 1);
  std::vector<C> gl(n2 * L);                                 // gl(j, ii) = gg_j^(ii+1)
  for (u64 j = 0; j < n2; ++j) {
    const C gg = std::exp(I * fm[j] * tau);
    for (int ii = 0; ii < L; ++ii) gl[j + n2 * ii] = std::pow(gg, (T)(ii + 1));
  }
  std::vector<C> glsum(L, C(0, 0));                          // sum(gl.t(), 1)
  for (int ii = 0; ii < L; ++ii)
    for (u64 j = 0; j < n2; ++j) glsum[ii] += std::conj(gl[j + n2 * ii]);
  CM<T> GTG((size_t)L * L, C(0, 0));
  for (int d = 0; d < L; ++d) GTG[(size_t)d * L + d] += (T)n2;
  for (int ii = 0; ii < L - 1; ++ii)
    for (int d = 0; d + ii + 1 < L; ++d) {
      GTG[(size_t)(d + ii + 1) * L + d] += glsum[ii];        // diag(-(ii+1))
      GTG[(size_t)d * L + (d + ii + 1)] += std::conj(glsum[ii]);
    }
  const T rcn = (T)1 / la_cond(GTG, L);
  CM<T> B;
  if (!(rcn > (T)(10 * 2e-16) && la_inverse(GTG, L, &B))) B = la_pinv(GTG, L);
  // iGTGGT = B * G^H, G columns: ones, then gl(:, 0 .. L-2)
  std::vector<C> P((size_t)L * n2, C(0, 0));
  for (int l = 0; l < L; ++l)
    for (u64 j = 0; j < n2; ++j) {
      C acc(0, 0);
      for (int k = 0; k < L; ++k) acc += B[(size_t)l * L + k] * std::conj(k == 0 ? C(1, 0) : gl[j + n2 * (k - 1)]);
      P[(size_t)l * n2 + j] = acc;
    }
  std::vector<C> AA(none * L), res(L);
  for (u64 m = 0; m < none; ++m) {                           // res = iGTGGT * exp(i fm t_m) (:140-145)
    std::fill(res.begin(), res.end(), C(0, 0));
    for (u64 j = 0; j < n2; ++j) {
      const C f = std::exp(I * fm[j] * tv[m]);
      for (int l = 0; l < L; ++l) res[l] += P[(size_t)l * n2 + j] * f;
    }
    for (int l = 0; l < L; ++l) AA[m + none * l] = std::conj(res[l]);
  }
  return AA;
}

// Histogram interpolator (TimeSegmentation.cpp:157-211) for one shot; the
// first L of its L+1 columns.  hist(X, 256) restates Armadillo 9.200's: bin
// centres min + (max - min) * (b + 0.5) / 256, nearest centre, ties low.
template <typename T>
std::vector<std::complex<T>> aa_histogram(const T* fm, u64 n2, const std::vector<T>& tv, u64 none, int L, T tau) {
  using C = std::complex<T>;
  const C I(0, 1);
  const int nbins = 256;
  T mn = fm[0], mx = fm[0];
  for (u64 j = 0; j < n2; ++j) { mn = std::min(mn, fm[j]); mx = std::max(mx, fm[j]); }
  std::vector<T> ctr(nbins);
  for (int b = 0; b < nbins; ++b) ctr[b] = (T)((0.5 + b) / (double)nbins);
  for (int b = 0; b < nbins; ++b) ctr[b] = (mx - mn) * ctr[b] + mn;
  std::vector<T> h(nbins, (T)0);
  for (u64 j = 0; j < n2; ++j) {
    int best = 0;
    T bd = std::abs(fm[j] - ctr[0]);
    for (int b = 1; b < nbins; ++b) {
      const T d = std::abs(fm[j] - ctr[b]);
      if (d < bd) { bd = d; best = b; } else { break; }
    }
    h[best] += (T)1;
  }
  const T rangeFM = mx - mn;
  const int KK = (int)std::floor(2.0 * kPiD / ((rangeFM / (T)nbins) * tau));
  if (KK < 2 * L + 1) throw std::runtime_error("oracle: histogram interpolator needs KK >= 2L+1");
  const T dwn = 2 * kPiD / (KK * tau);
  auto fft_k = [&](const std::vector<C>& in) {               // calcFFT1D(in, KK) (:225-242)
    std::vector<C> d(KK, C(0, 0));
    for (int b = 0; b < std::min(nbins, KK); ++b) d[b] = in[b];
    const std::size_t dims[1] = {(std::size_t)KK};
    fft_nd<T>(d.data(), dims, 1, -1);
    return d;
  };
  std::vector<C> temp(nbins);
  for (int b = 0; b < nbins; ++b) temp[b] = h[b] * std::exp(I * dwn * (T)b * tau * (T)L);
  std::vector<C> ftwe = fft_k(temp);
  for (int k = 0; k < KK; ++k) ftwe[k] = std::exp(-I * (mn + dwn / 2) * tau * ((T)k - (T)L)) * ftwe[k];
  const int n = L + 1;
  CM<T> At((size_t)n * n);                                   // GTGap_ap.st()
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) At[(size_t)r * n + c] = ftwe[L + r - c];
  CM<T> B;
  bool use_inv = la_inverse(At, n, &B);
  if (use_inv) use_inv = (T)1 / (la_norm1(At, n) * la_norm1(B, n)) > (T)(10 * std::numeric_limits<double>::epsilon());
  if (!use_inv) B = la_pinv(At, n);
  std::vector<C> AA(none * L);
  for (u64 m = 0; m < none; ++m) {
    for (int b = 0; b < nbins; ++b) temp[b] = h[b] * std::exp(I * (T)b * dwn * tv[m]);
    std::vector<C> ftc = fft_k(temp);
    for (int k = 0; k < n; ++k) ftc[k] = std::exp(I * (mn + dwn / 2) * (tv[m] - tau * (T)k)) * ftc[k];
    for (int l = 0; l < L; ++l) {
      C r(0, 0);
      for (int k = 0; k < n; ++k) r += B[(size_t)l * n + k] * ftc[k];
      AA[m + none * l] = std::conj(r);
    }
  }
  return AA;
}


// TimeSegmentation with the Hanning interpolator (TimeSegmentation.cpp:37-93,
// 213-218) and its operators (:252-324).  Holds a non-owning pointer to G,
// like the reference (TimeSegmentation.cpp:53).
template <typename T>
struct TimeSegOp : Op<T> {
  using C = std::complex<T>;
  const Op<T>* G;
  int L;
  u64 nshots;
  T tau, tmin;
  std::vector<C> AA;   // n1 x L, column-major (AA[m + n1*l])
  std::vector<C> Wo;   // n2 x (L+1)
  std::vector<C> WoH;

  TimeSegOp(const Op<T>* g, const T* fieldmap, const T* tvec, u64 a, u64 b, u64 nsegs, u64 interptype, u64 shots,
            bool tables64 = false)
      : G(g) {
    this->n1 = a; this->n2 = b;
    L = (nsegs == 0 || nsegs == 1) ? 1 : (int)nsegs;
    if (L > 1 && (interptype < 1 || interptype > 3)) throw std::runtime_error("oracle: interptype 1, 2 or 3");
    nshots = shots;
    std::vector<T> tv(tvec, tvec + a);
    T mn = *std::min_element(tv.begin(), tv.end());
    T mx = *std::max_element(tv.begin(), tv.end());
    tmin = mn;
    T rangt = mx - tmin;
    tau = (rangt + std::numeric_limits<double>::epsilon()) / L;
    for (auto& v : tv) v = v - tmin;
    const u64 none = a / shots;
    if (L <= 1) {
      L = 1; tau = 0;
      AA.assign(a * 2, C(1, 0));
      Wo.assign(b, C(1, 0));
      WoH.assign(b, C(1, 0));
    } else {
      std::vector<C> one(none * L);
      if (interptype == 1) {
        for (unsigned int l = 0; l < (unsigned)L; ++l)
          for (unsigned int m = 0; m < none; ++m) {
            if ((std::abs(tv[m] - ((l) * tau))) <= tau)
              one[m + none * l] = C(0.5 + 0.5 * std::cos((kPiD) * (tv[m] - ((l) * tau)) / tau), 0);
            else
              one[m + none * l] = C(0, 0);
          }
      } else if (tables64) {
        // the table built in double and rounded to T: the float gridding of
        // the reference with the interpolator of the FP64 path
        std::vector<double> fm64(fieldmap, fieldmap + b), tv64(tv.begin(), tv.end());
        const auto d = interptype == 2 ? aa_minmax<double>(fm64.data(), b, tv64, none, L, (double)tau)
                                       : aa_histogram<double>(fm64.data(), b, tv64, none, L, (double)tau);
        for (u64 q = 0; q < d.size(); ++q) one[q] = C((T)d[q].real(), (T)d[q].imag());
      } else if (interptype == 2) {
        one = aa_minmax<T>(fieldmap, b, tv, none, L, tau);
      } else {
        one = aa_histogram<T>(fieldmap, b, tv, none, L, tau);
      }
      AA.resize(a * L);
      for (int l = 0; l < L; ++l)
        for (u64 m = 0; m < a; ++m) AA[m + a * l] = one[(m % none) + none * l];
      Wo.resize(b * (L + 1));
      WoH.resize(b * (L + 1));
      for (unsigned int l = 0; l < (unsigned)L + 1; ++l) {
        T s = (l) * tau + tmin;
        for (u64 p = 0; p < b; ++p) {
          T v = fieldmap[p] * s;
          Wo[p + b * l] = C(std::cos(v), -std::sin(v));
          WoH[p + b * l] = C(std::cos(v), std::sin(v));
        }
      }
    }
  }
  void forward(const C* x, C* y) const override {
    const u64 n1 = this->n1, n2 = this->n2;
    std::vector<C> tmp(n2), out(n1);
    std::fill(y, y + n1, C(0, 0));
    for (int l = 0; l < L; ++l) {
      for (u64 p = 0; p < n2; ++p) tmp[p] = Wo[p + n2 * l] * x[p];
      G->forward(tmp.data(), out.data());
      for (u64 m = 0; m < n1; ++m) y[m] += out[m] * AA[m + n1 * l];
    }
  }
  void adjoint(const C* d, C* x) const override {
    const u64 n1 = this->n1, n2 = this->n2;
    std::vector<C> tmp(n1), img(n2);
    std::fill(x, x + n2, C(0, 0));
    for (int l = 0; l < L; ++l) {
      for (u64 m = 0; m < n1; ++m) tmp[m] = std::conj(AA[m + n1 * l]) * d[m];
      G->adjoint(tmp.data(), img.data());
      for (u64 p = 0; p < n2; ++p) x[p] += img[p] * WoH[p + n2 * l];
    }
  }
};

// SENSE coil loop (SENSE.cpp:33-97); non-owning pointer to G (SENSE.cpp:39).
template <typename T>
struct SenseOp : Op<T> {
  using C = std::complex<T>;
  const Op<T>* G;
  u64 nc;
  std::vector<C> S;  // n2 x nc
  SenseOp(const Op<T>* g, const C* smap, u64 a, u64 b, u64 c) : G(g), nc(c) {
    this->n1 = a; this->n2 = b;
    S.assign(smap, smap + b * c);
  }
  void forward(const C* x, C* y) const override {
    const u64 n1 = this->n1, n2 = this->n2;
    std::vector<C> tmp(n2);
    for (u64 c = 0; c < nc; ++c) {
      for (u64 p = 0; p < n2; ++p) tmp[p] = S[p + n2 * c] * x[p];
      G->forward(tmp.data(), y + n1 * c);
    }
  }
  void adjoint(const C* d, C* x) const override {
    const u64 n1 = this->n1, n2 = this->n2;
    std::vector<C> img(n2);
    std::fill(x, x + n2, C(0, 0));
    for (u64 c = 0; c < nc; ++c) {
      G->adjoint(d + n1 * c, img.data());
      for (u64 p = 0; p < n2; ++p) x[p] += img[p] * std::conj(S[p + n2 * c]);
    }
  }
};

template <typename T>
inline u64 op_data_len(const Op<T>& op) {
  if (auto* g = dynamic_cast<const GnufftOp<T>*>(&op)) return g->data_len();
  if (auto* s = dynamic_cast<const SenseOp<T>*>(&op)) return s->n1 * s->nc;
  return op.n1;
}

// pcSenseTimeSeg (pcSenseTimeSeg.cpp:41-171): per-shot Gnufft + TimeSegmentation.
template <typename T>
struct PcSenseTimeSegOp : Op<T> {
  using C = std::complex<T>;
  u64 Ni, Nc, Ns, Nd;
  std::vector<std::unique_ptr<GnufftOp<T>>> G;
  std::vector<std::unique_ptr<TimeSegOp<T>>> A;
  std::vector<C> M, Mc;  // Ni x (Nc*Ns), column s + c*Ns
  PcSenseTimeSegOp(const T* kx, const T* ky, const T* kz, u64 nk, int nx, int ny, int nz, u64 nc, const T* t,
                   u64 L, u64 type, const C* smap, const T* fmap, const T* pmap, u64 npmap, bool use_ref) {
    Ni = (u64)nx * ny * nz; Nc = nc; Ns = npmap / Ni; Nd = nk / Ns;
    this->n1 = Nd * Ns * Nc; this->n2 = Ni;
    for (u64 s = 0; s < Ns; ++s) {
      G.emplace_back(new GnufftOp<T>(Nd, (T)2.0, nx, ny, nz, kx + s * Nd, ky + s * Nd, kz + s * Nd));
      G.back()->use_ref = use_ref;
      A.emplace_back(new TimeSegOp<T>(G.back().get(), fmap, t + s * Nd, Nd, Ni, L, type, 1));
    }
    M.resize(Ni * Nc * Ns); Mc.resize(Ni * Nc * Ns);
    for (u64 c = 0; c < Nc; ++c)
      for (u64 s = 0; s < Ns; ++s)
        for (u64 p = 0; p < Ni; ++p) {
          T ph = pmap[p + Ni * s];
          C e(std::cos(ph), -std::sin(ph));
          M[p + Ni * (s + c * Ns)] = smap[p + Ni * c] * e;
          Mc[p + Ni * (s + c * Ns)] = std::conj(smap[p + Ni * c]) * std::conj(e);
        }
  }
  void forward(const C* x, C* y) const override {
    std::vector<C> tmp(Ni);
    for (u64 c = 0; c < Nc; ++c)
      for (u64 s = 0; s < Ns; ++s) {
        const C* m = M.data() + Ni * (s + c * Ns);
        for (u64 p = 0; p < Ni; ++p) tmp[p] = x[p] * m[p];
        A[s]->forward(tmp.data(), y + Nd * (s + c * Ns));
      }
  }
  void adjoint(const C* d, C* x) const override {
    std::vector<C> img(Ni);
    std::fill(x, x + Ni, C(0, 0));
    for (u64 c = 0; c < Nc; ++c)
      for (u64 s = 0; s < Ns; ++s) {
        A[s]->adjoint(d + Nd * (s + c * Ns), img.data());
        const C* m = Mc.data() + Ni * (s + c * Ns);
        for (u64 p = 0; p < Ni; ++p) x[p] += m[p] * img[p];
      }
  }
};

// pcSENSE (pcSENSE.cpp:40-153): per-shot Gdft over one voxel table.  The
// phase factor expiPMap = conj(exp(-i P)) = exp(+i P) (:103) weights both
// directions; the adjoint multiplies by conj(S) (.) expiPMap (:146).
template <typename T>
struct PcSenseOp : Op<T> {
  using C = std::complex<T>;
  u64 Ni, Nc, Ns, Nd;
  std::vector<T> ix, iy, iz;
  std::vector<std::unique_ptr<GdftOp<T>>> A;
  std::vector<C> S, E;  // Ni x Nc, Ni x Ns
  PcSenseOp(const T* kx, const T* ky, const T* kz, u64 nk, int nx, int ny, int nz, u64 nc, const T* t,
            const C* smap, const T* fmap, const T* pmap, u64 npmap, bool use_ref, bool exact64) {
    Ni = (u64)nx * ny * nz; Nc = nc; Ns = npmap / Ni; Nd = nk / Ns;
    this->n1 = Nd * Ns * Nc; this->n2 = Ni;
    // :65-82, cube (Nx, Ny, Nz) with y as its first index
    ix.resize(Ni); iy.resize(Ni); iz.resize(Ni);
    for (int ii = 0; ii < ny; ++ii)
      for (int jj = 0; jj < nx; ++jj)
        for (int kk = 0; kk < nz; ++kk) {
          const u64 j = (u64)ii + (u64)nx * jj + (u64)nx * ny * kk;
          ix[j] = (T)(((T)jj - (T)nx / 2.0) / ((T)nx));
          iy[j] = (T)(((T)ii - (T)ny / 2.0) / ((T)ny));
          iz[j] = (T)(((T)kk - (T)nz / 2.0) / ((T)nz));
        }
    for (u64 s = 0; s < Ns; ++s) {
      A.emplace_back(new GdftOp<T>(Nd, Ni, kx + s * Nd, ky + s * Nd, kz + s * Nd, ix.data(), iy.data(), iz.data(),
                                   fmap, t + s * Nd));
      A.back()->use_ref = use_ref;
      A.back()->exact64 = exact64;
    }
    S.assign(smap, smap + Ni * Nc);
    E.resize(Ni * Ns);
    for (u64 i = 0; i < Ni * Ns; ++i) E[i] = std::conj(std::exp(C(0, -1) * pmap[i]));
  }
  void forward(const C* x, C* y) const override {
    std::vector<C> tmp(Ni);
    for (u64 c = 0; c < Nc; ++c)
      for (u64 s = 0; s < Ns; ++s) {
        for (u64 p = 0; p < Ni; ++p) tmp[p] = x[p] * (S[p + Ni * c] * E[p + Ni * s]);
        A[s]->forward(tmp.data(), y + Nd * (s + c * Ns));
      }
  }
  void adjoint(const C* d, C* x) const override {
    std::vector<C> img(Ni);
    std::fill(x, x + Ni, C(0, 0));
    for (u64 c = 0; c < Nc; ++c)
      for (u64 s = 0; s < Ns; ++s) {
        A[s]->adjoint(d + Nd * (s + c * Ns), img.data());
        for (u64 p = 0; p < Ni; ++p) x[p] += (std::conj(S[p + Ni * c]) * E[p + Ni * s]) * img[p];
      }
  }
};

// LRobj (lowRank/LRobj.cpp:27-68): the partial-separability model.  x = vec(X)
// with X N x K (K = rank); operator* forms the images X v (v: K x Nimg,
// column-major) and sends image i through A_all[i] (:39-50); operator/ applies
// A_all[i] / d_i and multiplies the N x Nimg stack by trans(v) (conjugate
// transpose, :53-66).  The per-image operators are borrowed, as the reference
// holds raw pointers.
template <typename T>
struct LowRankOp : Op<T> {
  using C = std::complex<T>;
  u64 N, Nd, K, Ni;
  std::vector<C> v;
  std::vector<const Op<T>*> A;
  LowRankOp(u64 n, u64 nd, u64 k, u64 ni, const C* vb, std::vector<const Op<T>*> ops)
      : N(n), Nd(nd), K(k), Ni(ni), v(vb, vb + k * ni), A(std::move(ops)) {
    if (A.size() != Ni) throw std::runtime_error("LRobj: one operator per image");
    for (const Op<T>* a : A)
      if (op_image_len(*a) != N || op_data_len(*a) != Nd)
        throw std::runtime_error("LRobj: operator sizes differ from NimgSize / N_data");
    this->n1 = Nd * Ni;
    this->n2 = N * K;
  }
  void forward(const C* x, C* y) const override {
    std::vector<C> img(N);
    for (u64 i = 0; i < Ni; ++i) {
      std::fill(img.begin(), img.end(), C(0, 0));
      for (u64 k = 0; k < K; ++k) {
        const C c = v[k + K * i];
        for (u64 p = 0; p < N; ++p) img[p] += x[p + N * k] * c;
      }
      A[i]->forward(img.data(), y + Nd * i);
    }
  }
  void adjoint(const C* d, C* x) const override {
    std::vector<C> img(N * Ni);
    for (u64 i = 0; i < Ni; ++i) A[i]->adjoint(d + Nd * i, img.data() + N * i);
    std::fill(x, x + N * K, C(0, 0));
    for (u64 k = 0; k < K; ++k)
      for (u64 i = 0; i < Ni; ++i) {
        const C c = std::conj(v[k + K * i]);
        for (u64 p = 0; p < N; ++p) x[p + N * k] += img[p + N * i] * c;
      }
  }
};

// ---------------------------------------------------------------------------
// Regularizers (Robject.cpp:49-193, QuadPenalty.cpp:45-64, TVPenalty.cpp:43-68)
// ---------------------------------------------------------------------------
template <typename T>
struct Penalty {
  using C = std::complex<T>;
  int kind = 0;  // 0 quadratic, 1 TV
  u64 Nx = 1, Ny = 1, Nz = 1;
  T beta = 0, delta = 1;
  u64 dims2pen = 3;
  u64 nd() const { return (Nz == 1 || dims2pen == 2) ? 2 : 3; }
  u64 offset(u64 dim) const { return dim == 0 ? 1 : dim == 1 ? Ny : Nx * Ny; }

  // Cd: out[i] = d[i] - d[i-off] for i >= off, else 0 (Robject.cpp:76-79).
  void Cd(const C* d, u64 dim, C* out) const {
    const u64 N = Nx * Ny * Nz, off = offset(dim);
    std::fill(out, out + N, C(0, 0));
    for (u64 i = off; i < N; ++i) out[i] = d[i] - d[i - off];
  }
  // Ctd exactly as Robject.cpp:111-117 (not the exact adjoint of Cd).
  void Ctd(const C* d, u64 dim, C* out) const {
    const u64 N = Nx * Ny * Nz, off = offset(dim);
    std::fill(out, out + N, C(0, 0));
    out[off - 1] = -d[off];
    out[N - 1 - off] = d[N - 1 - off];
    for (u64 i = off; i < N - 1; ++i) out[i - off] = d[i - off] - d[i];
  }
  C wpot(C d) const {
    if (kind == 0) return C(1, 0);
    T a = std::abs(d / delta);
    return C((T)1 / std::sqrt((T)1 + a * a), 0);
  }
  C dpot(C d) const {
    if (kind == 0) return d;
    T a = std::abs(d / delta);
    return d / std::sqrt((T)1 + a * a);
  }
  void Gradient(const C* x, C* g) const {
    const u64 N = Nx * Ny * Nz;
    std::vector<C> d(N), e(N);
    std::fill(g, g + N, C(0, 0));
    for (u64 dim = 0; dim < nd(); ++dim) {
      Cd(x, dim, d.data());
      for (u64 i = 0; i < N; ++i) d[i] = dpot(d[i]);
      Ctd(d.data(), dim, e.data());
      for (u64 i = 0; i < N; ++i) g[i] += e[i];
    }
    for (u64 i = 0; i < N; ++i) g[i] = beta * g[i];
  }
  C Denom(const C* ddir, const C* x) const {
    const u64 N = Nx * Ny * Nz;
    std::vector<C> cdir(N), cx(N);
    C pen(0, 0);
    for (u64 dim = 0; dim < nd(); ++dim) {
      Cd(ddir, dim, cdir.data());
      Cd(x, dim, cx.data());
      C acc(0, 0);
      for (u64 i = 0; i < N; ++i) acc += std::conj(cdir[i]) * (wpot(cx[i]) * cdir[i]);
      pen += acc;
    }
    return pen * C(beta, 0);
  }
};

// R_lowRank (lowRank/R_lowRank.cpp:27-95) over a Robject R.  With x = vec(X),
// X N x K, it penalises the columns of I = X * trans(v.cols(0, K-1)) (:42-44;
// trans is the conjugate transpose, so I[n, j] = sum_k X[n, k] conj(v[j, k])).
// Gradient (:50-64) returns vectorise(strans(v.cols(0, K-1)) * strans(Y)) with
// Y_j = R.Gradient(I_j): a K x N matrix, element [k + K*n].  That product is
// defined only when K == Nimg (K x K times Nimg x N), so v here is K x K.
// Denom (:67-87) is R.Beta * sum_j R.Denom(D_j, I_j), D = Ddir * trans(v), and
// R.Denom already carries one factor beta.
template <typename T>
struct LowRankPenalty {
  using C = std::complex<T>;
  const Penalty<T>* R = nullptr;
  u64 K = 1;
  std::vector<C> v;   // K x K, column-major
  u64 n() const { return R->Nx * R->Ny * R->Nz; }
  void mix(const C* x, C* I) const {
    const u64 N = n();
    std::fill(I, I + N * K, C(0, 0));
    for (u64 j = 0; j < K; ++j)
      for (u64 k = 0; k < K; ++k) {
        const C c = std::conj(v[j + K * k]);
        for (u64 p = 0; p < N; ++p) I[p + N * j] += x[p + N * k] * c;
      }
  }
  void Gradient(const C* x, C* g) const {
    const u64 N = n();
    std::vector<C> I(N * K), Y(N * K);
    mix(x, I.data());
    for (u64 j = 0; j < K; ++j) R->Gradient(I.data() + N * j, Y.data() + N * j);
    for (u64 p = 0; p < N; ++p)
      for (u64 k = 0; k < K; ++k) {
        C acc(0, 0);
        for (u64 j = 0; j < K; ++j) acc += v[j + K * k] * Y[p + N * j];
        g[k + K * p] = acc;
      }
  }
  C Denom(const C* ddir, const C* x) const {
    const u64 N = n();
    std::vector<C> I(N * K), D(N * K);
    mix(x, I.data());
    mix(ddir, D.data());
    C sum(0, 0);
    for (u64 j = 0; j < K; ++j) sum += R->Denom(D.data() + N * j, I.data() + N * j);
    return R->beta * sum;
  }
};

template <typename T>
inline std::complex<T> cdot(const std::complex<T>* a, const std::complex<T>* b, u64 n) {
  std::complex<T> s(0, 0);
  for (u64 i = 0; i < n; ++i) s += std::conj(a[i]) * b[i];
  return s;
}

// solve_pwls_pcg (solve_pwls_pcg.hpp:48-167), scalars complex<T> as in the reference.
// Returns the number of completed iterations.
template <typename T, typename Robj>
int pwls_pcg(const Op<T>& A, const std::complex<T>* x0, const T* W, const std::complex<T>* y,
             const Robj& R, u64 niter, std::complex<T>* xout) {
  using C = std::complex<T>;
  const u64 nd = op_data_len(A), ni = op_image_len(A);
  std::vector<C> x(x0, x0 + ni), Ax(nd), r(nd), ngrad(ni), ddir(ni, C(0, 0)), Adir(nd), pgrad(ni), xs(ni);
  A.forward(x.data(), Ax.data());
  C oldinprod = 0, gamma = 0;
  // norm_grad denominator real(y' * (W % y)) (solve_pwls_pcg.hpp:42-46)
  T ywy = 0;
  {
    C s(0, 0);
    for (u64 m = 0; m < nd; ++m) s += std::conj(y[m]) * (W[m] * y[m]);
    ywy = s.real();
  }
  int done = 0;
  for (u64 it = 0; it < niter; ++it) {
    for (u64 m = 0; m < nd; ++m) r[m] = W[m] * (y[m] - Ax[m]);
    A.adjoint(r.data(), ngrad.data());
    T gn = 0;
    for (u64 j = 0; j < ni; ++j) gn += std::norm(ngrad[j]);
    if (std::sqrt(gn) / ywy < 1e-10) break;
    R.Gradient(x.data(), pgrad.data());
    for (u64 j = 0; j < ni; ++j) ngrad[j] -= pgrad[j];
    C newinprod = cdot(ngrad.data(), ngrad.data(), ni).real();
    if (it == 0) {
      ddir = ngrad;
    } else {
      gamma = (std::abs(oldinprod) < 1e-10) ? C(0, 0) : newinprod / oldinprod;
      for (u64 j = 0; j < ni; ++j) ddir[j] = ngrad[j] + gamma * ddir[j];
    }
    oldinprod = newinprod;
    if (cdot(ddir.data(), ngrad.data(), ni).real() < 0) break;
    A.forward(ddir.data(), Adir.data());
    C dAWAd = 0, dAWr = 0;
    {
      C s1(0, 0), s2(0, 0);
      for (u64 m = 0; m < nd; ++m) {
        s1 += std::conj(Adir[m]) * (W[m] * Adir[m]);
        s2 += std::conj(Adir[m]) * (W[m] * (y[m] - Ax[m]));
      }
      dAWAd = s1.real();
      dAWr = s2.real();
    }
    C step = 0;
    bool stop = false;
    for (int j = 0; j < 3; ++j) {
      for (u64 p = 0; p < ni; ++p) xs[p] = x[p] + step * ddir[p];
      C pdenom = R.Denom(ddir.data(), xs.data());
      C denom = dAWAd + pdenom;
      if (std::abs(denom) < 1e-20 || std::abs(denom) > 1e25) { stop = true; break; }
      R.Gradient(xs.data(), pgrad.data());
      C pdot = cdot(ddir.data(), pgrad.data(), ni).real();
      step -= (-dAWr + step * dAWAd + pdot) / denom;
    }
    if (stop) break;
    for (u64 m = 0; m < nd; ++m) Ax[m] += step * Adir[m];
    for (u64 p = 0; p < ni; ++p) x[p] += step * ddir[p];
    done = (int)it + 1;
  }
  std::copy(x.begin(), x.end(), xout);
  return done;
}

}  // namespace pgo
