// ORACLE / TEST INFRASTRUCTURE ONLY — never linked into the product library.
//
// CPU FFT engine used by the oracle in two places:
//   * behind the FFTW-API shim (fftw_shim/), so the reference's own
//     PowerGrid/fftCPU.cpp (which calls fftwf_plan_dft_{1,2,3}d / fftw_execute,
//     fftCPU.cpp:35-176) links and runs here although FFTW 3 is not installed;
//   * directly by the restated Gnufft pipeline (pg_oracle.hpp).
//
// Semantics follow FFTW's documented conventions: unnormalised complex DFT,
// X[k] = sum_j x[j] * exp(sign * 2*pi*i*j*k/n) with sign = -1 (FFTW_FORWARD)
// or +1 (FFTW_BACKWARD); multi-dimensional plans are row-major (the last
// dimension varies fastest).
//
// Algorithm: mixed-radix Stockham autosort (decimation in frequency), radices
// 4, 2, 3, 5 and a direct DFT stage for any remaining prime factor.  A
// transform along a slow dimension runs as interleaved transforms whose
// innermost loop is contiguous in memory, so every pass streams.  Twiddles
// are computed in double precision and rounded to T.
#pragma once

#include <cmath>
#include <complex>
#include <cstddef>
#include <cstring>
#include <vector>

namespace pgo {

template <typename T>
class FftStockham {
 public:
  using C = std::complex<T>;

  FftStockham(std::size_t n, int sign) : n_(n), sign_(sign) { plan(); }

  std::size_t size() const { return n_; }

  // Transforms `inner` interleaved sequences of length n stored as
  // data[q + inner * i], q < inner, i < n.  `scratch` must hold n*inner.
  void exec(C* data, std::size_t inner, C* scratch) const {
    if (n_ <= 1) return;
    C* x = data;
    C* y = scratch;
    std::size_t s = inner;   // current stride
    std::size_t len = n_;    // current sub-transform length
    for (const Stage& st : stages_) {
      run_stage(st, len, s, x, y);
      len /= st.radix;
      s *= st.radix;
      C* t = x; x = y; y = t;
    }
    if (x != data) std::memcpy(data, x, sizeof(C) * n_ * inner);
  }

 private:
  struct Stage {
    std::size_t radix;
    std::size_t m;               // len / radix for this stage
    std::vector<C> tw;           // tw[p*radix + k] = exp(sign*2*pi*i*p*k/len)
    std::vector<C> rootr;        // exp(sign*2*pi*i*j/radix), j < radix
  };

  void plan() {
    std::size_t len = n_;
    while (len > 1) {
      std::size_t r = 0;
      if (len % 4 == 0) r = 4;
      else if (len % 2 == 0) r = 2;
      else if (len % 3 == 0) r = 3;
      else if (len % 5 == 0) r = 5;
      else {
        for (std::size_t f = 7; f * f <= len; f += 2)
          if (len % f == 0) { r = f; break; }
        if (r == 0) r = len;  // prime remainder: one direct-DFT stage
      }
      Stage st;
      st.radix = r;
      st.m = len / r;
      st.tw.resize(st.m * r);
      const double two_pi = 6.283185307179586476925286766559;
      for (std::size_t p = 0; p < st.m; ++p)
        for (std::size_t k = 0; k < r; ++k) {
          const std::size_t e = (p * k) % len;
          const double ang = sign_ * two_pi * static_cast<double>(e) / static_cast<double>(len);
          st.tw[p * r + k] = C(static_cast<T>(std::cos(ang)), static_cast<T>(std::sin(ang)));
        }
      st.rootr.resize(r);
      for (std::size_t j = 0; j < r; ++j) {
        const double ang = sign_ * two_pi * static_cast<double>(j) / static_cast<double>(r);
        st.rootr[j] = C(static_cast<T>(std::cos(ang)), static_cast<T>(std::sin(ang)));
      }
      stages_.push_back(st);
      len /= r;
    }
  }

  // One Stockham DIF pass: for p < m, q < s:
  //   a_j = x[q + s*(p + j*m)],  y[q + s*(r*p + k)] = (sum_j a_j w_r^{jk}) * w_len^{pk}
  void run_stage(const Stage& st, std::size_t len, std::size_t s, const C* x, C* y) const {
    const std::size_t r = st.radix, m = st.m;
    (void)len;
    const T sg = static_cast<T>(sign_);
    if (r == 2) {
      for (std::size_t p = 0; p < m; ++p) {
        const C w1 = st.tw[p * 2 + 1];
        const C* x0 = x + s * p;
        const C* x1 = x + s * (p + m);
        C* y0 = y + s * (2 * p);
        C* y1 = y + s * (2 * p + 1);
        for (std::size_t q = 0; q < s; ++q) {
          const C a = x0[q], b = x1[q];
          y0[q] = a + b;
          y1[q] = (a - b) * w1;
        }
      }
    } else if (r == 4) {
      for (std::size_t p = 0; p < m; ++p) {
        const C w1 = st.tw[p * 4 + 1], w2 = st.tw[p * 4 + 2], w3 = st.tw[p * 4 + 3];
        const C* x0 = x + s * p;
        const C* x1 = x + s * (p + m);
        const C* x2 = x + s * (p + 2 * m);
        const C* x3 = x + s * (p + 3 * m);
        C* y0 = y + s * (4 * p);
        C* y1 = y + s * (4 * p + 1);
        C* y2 = y + s * (4 * p + 2);
        C* y3 = y + s * (4 * p + 3);
        for (std::size_t q = 0; q < s; ++q) {
          const C a0 = x0[q], a1 = x1[q], a2 = x2[q], a3 = x3[q];
          const C t0 = a0 + a2, t1 = a0 - a2;
          const C t2 = a1 + a3;
          const C d = a1 - a3;
          // multiply d by (sign * i)
          const C t3(-sg * d.imag(), sg * d.real());
          y0[q] = t0 + t2;
          y1[q] = (t1 + t3) * w1;
          y2[q] = (t0 - t2) * w2;
          y3[q] = (t1 - t3) * w3;
        }
      }
    } else {
      std::vector<C> a(r), b(r);
      for (std::size_t p = 0; p < m; ++p) {
        for (std::size_t q = 0; q < s; ++q) {
          for (std::size_t j = 0; j < r; ++j) a[j] = x[q + s * (p + j * m)];
          for (std::size_t k = 0; k < r; ++k) {
            C acc = a[0];
            for (std::size_t j = 1; j < r; ++j) acc += a[j] * st.rootr[(j * k) % r];
            b[k] = acc;
          }
          for (std::size_t k = 0; k < r; ++k) y[q + s * (r * p + k)] = b[k] * st.tw[p * r + k];
        }
      }
    }
  }

  std::size_t n_;
  int sign_;
  std::vector<Stage> stages_;
};

// In-place N-dimensional transform over row-major dims (dims[rank-1] fastest).
template <typename T>
void fft_nd(std::complex<T>* data, const std::size_t* dims, int rank, int sign) {
  std::size_t total = 1;
  for (int d = 0; d < rank; ++d) total *= dims[d];
  if (total <= 1) return;
  std::vector<std::complex<T>> scratch(total);
  std::size_t inner = 1;
  for (int d = rank - 1; d >= 0; --d) {
    const std::size_t n = dims[d];
    const std::size_t outer = total / (n * inner);
    if (n > 1) {
      FftStockham<T> f(n, sign);
      for (std::size_t o = 0; o < outer; ++o)
        f.exec(data + o * n * inner, inner, scratch.data());
    }
    inner *= n;
  }
}

}  // namespace pgo
