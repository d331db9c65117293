// Time-segmentation interpolators other than Hanning: the exact least-squares
// min-max interpolator (TimeSegmentation.cpp:94-156, interptype 2) and its
// histogram approximation (TimeSegmentation.cpp:157-211, interptype 3).
//
// Both are one-off host tables, as in the reference, computed here in double
// precision: the Gram matrices they invert are Toeplitz matrices of
// exponentials whose condition number grows quickly with L (about 1e12 at
// L = 8 over a +-100 Hz field map), so single precision leaves the table
// dominated by rounding.  The small dense algebra (LU inverse, one-sided
// Jacobi SVD for the condition number and the pseudo-inverse) is written out
// below; the sample loops run on all host threads.
#include <algorithm>
#include <cmath>
#include <complex>
#include <thread>
#include <vector>

#include "pg_ops.cuh"

namespace pg {
namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.141592653589793238462643383279502884;

struct CMat {
  int n = 0;
  std::vector<cd> a;  // row-major
  explicit CMat(int m = 0) : n(m), a((size_t)m * m) {}
  cd& operator()(int r, int c) { return a[(size_t)r * n + c]; }
  cd operator()(int r, int c) const { return a[(size_t)r * n + c]; }
};

// Gauss-Jordan inverse with partial pivoting; false if a pivot is exactly 0.
bool inverse(CMat A, CMat* out) {
  const int n = A.n;
  CMat I(n);
  for (int i = 0; i < n; ++i) I(i, i) = 1.0;
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::abs(A(r, c)) > std::abs(A(p, c))) p = r;
    if (A(p, c) == cd(0)) return false;
    if (p != c)
      for (int k = 0; k < n; ++k) {
        std::swap(A(p, k), A(c, k));
        std::swap(I(p, k), I(c, k));
      }
    const cd inv = 1.0 / A(c, c);
    for (int k = 0; k < n; ++k) {
      A(c, k) *= inv;
      I(c, k) *= inv;
    }
    for (int r = 0; r < n; ++r) {
      if (r == c || A(r, c) == cd(0)) continue;
      const cd f = A(r, c);
      for (int k = 0; k < n; ++k) {
        A(r, k) -= f * A(c, k);
        I(r, k) -= f * I(c, k);
      }
    }
  }
  *out = I;
  return true;
}

// One-sided Jacobi SVD A = U diag(s) V^H (Hestenes), square complex A.
void svd(const CMat& A, std::vector<double>* s, CMat* U, CMat* V) {
  const int n = A.n;
  CMat W = A;  // columns converge to U * s
  CMat Vm(n);
  for (int i = 0; i < n; ++i) Vm(i, i) = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double app = 0, aqq = 0;
        cd apq = 0;
        for (int i = 0; i < n; ++i) {
          app += std::norm(W(i, p));
          aqq += std::norm(W(i, q));
          apq += std::conj(W(i, p)) * W(i, q);
        }
        const double mag = std::abs(apq);
        if (mag == 0.0 || mag <= 1e-15 * std::sqrt(app * aqq)) continue;
        off = std::max(off, mag / std::sqrt(app * aqq));
        // rotate columns p, q to make them orthogonal
        const cd ph = apq / mag;
        const double tau = (aqq - app) / (2.0 * mag);
        const double t = (tau >= 0 ? 1.0 : -1.0) / (std::abs(tau) + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t), sn = c * t;
        for (int i = 0; i < n; ++i) {
          const cd wp = W(i, p), wq = W(i, q);
          W(i, p) = c * wp - sn * std::conj(ph) * wq;
          W(i, q) = sn * ph * wp + c * wq;
          const cd vp = Vm(i, p), vq = Vm(i, q);
          Vm(i, p) = c * vp - sn * std::conj(ph) * vq;
          Vm(i, q) = sn * ph * vp + c * vq;
        }
      }
    if (off < 1e-15) break;
  }
  s->assign(n, 0.0);
  CMat Um(n);
  for (int j = 0; j < n; ++j) {
    double nr = 0;
    for (int i = 0; i < n; ++i) nr += std::norm(W(i, j));
    nr = std::sqrt(nr);
    (*s)[j] = nr;
    for (int i = 0; i < n; ++i) Um(i, j) = nr > 0 ? W(i, j) / nr : cd(0);
  }
  *U = Um;
  *V = Vm;
}

// Moore-Penrose pseudo-inverse, singular values below n * max(s) * eps
// dropped (Armadillo's default tolerance).
CMat pinv(const CMat& A) {
  const int n = A.n;
  std::vector<double> s;
  CMat U, V;
  svd(A, &s, &U, &V);
  const double smax = *std::max_element(s.begin(), s.end());
  const double tol = n * smax * std::numeric_limits<double>::epsilon();
  CMat P(n);
  for (int k = 0; k < n; ++k) {
    if (s[k] <= tol) continue;
    const double inv = 1.0 / s[k];
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c) P(r, c) += V(r, k) * inv * std::conj(U(c, k));
  }
  return P;
}

double cond2(const CMat& A) {
  std::vector<double> s;
  CMat U, V;
  svd(A, &s, &U, &V);
  const double smax = *std::max_element(s.begin(), s.end());
  const double smin = *std::min_element(s.begin(), s.end());
  return smin > 0 ? smax / smin : std::numeric_limits<double>::infinity();
}

double norm1(const CMat& A) {
  double m = 0;
  for (int c = 0; c < A.n; ++c) {
    double s = 0;
    for (int r = 0; r < A.n; ++r) s += std::abs(A(r, c));
    m = std::max(m, s);
  }
  return m;
}

// Inverse, or the pseudo-inverse when the matrix is too ill-conditioned for
// one (the reference's branch, with its threshold).
CMat invert(const CMat& A, bool use_inverse) {
  CMat B;
  if (use_inverse && inverse(A, &B)) return B;
  return pinv(A);
}

// Run f(m) for m in [0, n) on all host threads.
template <typename F>
void parallel_for(uint64_t n, F f) {
  unsigned nt = std::max(1u, std::thread::hardware_concurrency());
  nt = (unsigned)std::min<uint64_t>(nt, std::max<uint64_t>(1, n / 64));
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (uint64_t m = t; m < n; m += nt) f(m);
    });
  for (auto& x : th) x.join();
}

}  // namespace

// Exact LS (min-max) interpolator, TimeSegmentation.cpp:94-156.  G (n2 x L)
// has columns exp(i*k*fm*tau), k < L; AA(m, l) = conj((GTG^-1 G^H f_m)_l)
// with f_m = exp(i*fm*t_m).
pg_status ts_aa_minmax(const float* fm, uint64_t n2, const std::vector<float>& tv, int L, float tau,
                       std::vector<float2>* aa) {
  const uint64_t none = tv.size();
  // glsum(k) = sum_j conj(exp(i*(k+1)*fm_j*tau)); GTG Hermitian Toeplitz (:116-126)
  std::vector<cd> glsum(L, 0.0);
  for (uint64_t j = 0; j < n2; ++j)
    for (int k = 0; k < L; ++k) glsum[k] += std::polar(1.0, -(double)(k + 1) * (double)fm[j] * (double)tau);
  CMat GTG(L);
  for (int r = 0; r < L; ++r)
    for (int c = 0; c < L; ++c)
      GTG(r, c) = r == c ? cd((double)n2) : r > c ? glsum[r - c - 1] : std::conj(glsum[c - r - 1]);
  const double rcn = 1.0 / cond2(GTG);
  const CMat B = invert(GTG, rcn > 10 * 2e-16);  // :128-133
  // iGTGGT(l, j) = sum_k B(l, k) exp(-i*k*fm_j*tau)
  std::vector<cd> P((size_t)L * n2);
  for (uint64_t j = 0; j < n2; ++j)
    for (int l = 0; l < L; ++l) {
      cd s = 0;
      for (int k = 0; k < L; ++k) s += B(l, k) * std::polar(1.0, -(double)k * (double)fm[j] * (double)tau);
      P[(size_t)l * n2 + j] = s;
    }
  aa->assign(none * L, make_float2(0.f, 0.f));
  parallel_for(none, [&](uint64_t m) {  // :140-145
    std::vector<cd> res(L, 0.0);
    const double t = tv[m];
    for (uint64_t j = 0; j < n2; ++j) {
      const cd f = std::polar(1.0, (double)fm[j] * t);
      for (int l = 0; l < L; ++l) res[l] += P[(size_t)l * n2 + j] * f;
    }
    for (int l = 0; l < L; ++l) (*aa)[m + none * l] = make_float2((float)res[l].real(), (float)-res[l].imag());
  });
  return PG_OK;
}

// Histogram (approximate min-max) interpolator, TimeSegmentation.cpp:157-211.
pg_status ts_aa_histogram(const float* fm, uint64_t n2, const std::vector<float>& tv, int L, float tau,
                          std::vector<float2>* aa) {
  const uint64_t none = tv.size();
  const int nbins = 256;
  // Armadillo hist(X, 256): bin centres min + (max - min) * (b + 0.5) / 256,
  // each value counted in its nearest centre (ties to the lower bin); the
  // first and last bins are open-ended.
  float mn = fm[0], mx = fm[0];
  for (uint64_t j = 0; j < n2; ++j) {
    mn = std::min(mn, fm[j]);
    mx = std::max(mx, fm[j]);
  }
  std::vector<float> centre(nbins);
  for (int b = 0; b < nbins; ++b) centre[b] = (float)((0.5 + b) / (double)nbins);
  for (int b = 0; b < nbins; ++b) centre[b] = (mx - mn) * centre[b] + mn;
  std::vector<double> h(nbins, 0.0);
  for (uint64_t j = 0; j < n2; ++j) {
    const float v = fm[j];
    int best = 0;
    float bd = std::abs(v - centre[0]);
    for (int b = 1; b < nbins; ++b) {
      const float d = std::abs(v - centre[b]);
      if (d < bd) { bd = d; best = b; } else { break; }
    }
    h[best] += 1.0;
  }
  // KK and dwn with the reference's operand types (:171-175)
  const float rangeFM = mx - mn;
  if (!(rangeFM > 0.f))
    return set_error(PG_INVALID_ARG, "TimeSegmentation: histogram interpolator needs a non-constant field map");
  const int KK = (int)std::floor(2.0 * kPi / ((rangeFM / (float)nbins) * tau));
  if (KK < 2 * L + 1)
    return set_error(PG_INVALID_ARG, "TimeSegmentation: histogram interpolator needs %d >= 2L+1 frequency bins", KK);
  const float dwn = (float)(2 * kPi / (float)(KK * tau));
  const int nb = std::min(nbins, KK);  // calcFFT1D trims to KK points (:225-236)
  const double off = (double)mn + (double)dwn / 2.0;
  // GTG approximation: ftwe(k) for k <= 2L (:177-185)
  std::vector<cd> ftwe(2 * L + 1);
  for (int k = 0; k <= 2 * L; ++k) {
    cd s = 0;
    for (int b = 0; b < nb; ++b)
      s += h[b] * std::polar(1.0, (double)dwn * b * (double)tau * L - 2.0 * kPi * (double)b * k / KK);
    ftwe[k] = std::polar(1.0, -off * (double)tau * (double)(k - L)) * s;
  }
  // GTGap(r, c) = ftwe(L + c - r); the reference inverts its plain transpose (:187-194)
  const int n = L + 1;
  CMat At(n);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) At(r, c) = ftwe[L + r - c];
  CMat Ai;
  bool use_inv = inverse(At, &Ai);
  if (use_inv) {
    const double rc = 1.0 / (norm1(At) * norm1(Ai));  // rcond in the 1-norm
    use_inv = rc > 10 * std::numeric_limits<double>::epsilon();
  }
  const CMat B = use_inv ? Ai : pinv(At);
  aa->assign(none * L, make_float2(0.f, 0.f));
  parallel_for(none, [&](uint64_t m) {  // :197-206
    const double t = tv[m];
    std::vector<cd> gtc(n);
    for (int k = 0; k < n; ++k) {
      cd s = 0;
      for (int b = 0; b < nb; ++b) s += h[b] * std::polar(1.0, (double)b * (double)dwn * t - 2.0 * kPi * (double)b * k / KK);
      gtc[k] = std::polar(1.0, off * (t - (double)tau * k)) * s;
    }
    for (int l = 0; l < L; ++l) {  // the first L of the L+1 columns are applied (:266-323)
      cd r = 0;
      for (int k = 0; k < n; ++k) r += B(l, k) * gtc[k];
      (*aa)[m + none * l] = make_float2((float)r.real(), (float)-r.imag());
    }
  });
  return PG_OK;
}

}  // namespace pg
