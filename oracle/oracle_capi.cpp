// ORACLE / TEST INFRASTRUCTURE ONLY — loaded by tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg, never by the product library.
//
// extern "C" surface over pg_oracle.hpp for ctypes.  Precision codes:
//   0  float  — the reference CPU path (T1 = float)
//   1  double — the reference's double instantiation (ftCpu<double> keeps sinf/cosf)
//   2  FP64   — the FP64 oracle (as 1, but the DFT evaluates sin/cos in double)
//   3  FP64 evaluation of the float Gnufft: window bounds, LUT index, LUT
//      values and beta as the float instantiation computes them, every other
//      step in double (the float operator without its rounding)
// All geometry / map / time inputs arrive as float32 (what the product
// receives) and are widened for precision 1/2.  Complex vectors are
// interleaved complex64 for precision 0 and complex128 otherwise.
//
// orc_use_reference() switches Gnufft and Gdft (precision 0/1) onto the
// reference's own compiled kernels in oracle/_ref/libpgref.so; composites,
// regularizers and PCG stay the restatement (the reference's versions need
// Armadillo, which is absent).
#include <dlfcn.h>

#include <atomic>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "pg_oracle.hpp"

using pgo::u64;

namespace {

bool g_use_ref = false;
int g_threads = 1;
thread_local bool t_in_worker = false;
std::string g_err;

template <typename F>
void parallel_for(u64 n, F fn) {
  const int nt = (int)std::min<u64>((u64)std::max(1, g_threads), n);
  if (nt <= 1 || t_in_worker) {
    for (u64 i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<u64> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&]() {
      t_in_worker = true;
      for (u64 i; (i = next.fetch_add(1)) < n;) fn(i);
      t_in_worker = false;
    });
  for (auto& x : th) x.join();
}

// SENSE<TimeSegmentation<G>> with the (coil, segment) loop flattened over
// threads.  Per-element arithmetic and summation order equal the nested
// serial loops of SENSE.cpp:51-97 and TimeSegmentation.cpp:252-324.
template <typename T>
struct SenseParallel : pgo::SenseOp<T> {
  using C = std::complex<T>;
  using pgo::SenseOp<T>::SenseOp;
  void forward(const C* x, C* y) const override {
    auto* ts = dynamic_cast<const pgo::TimeSegOp<T>*>(this->G);
    if (!ts || g_threads <= 1) return pgo::SenseOp<T>::forward(x, y);
    const u64 n1 = this->n1, n2 = this->n2, L = ts->L, nc = this->nc;
    std::vector<C> out(n1 * L * nc);
    parallel_for(nc * L, [&](u64 u) {
      const u64 c = u / L, l = u % L;
      std::vector<C> tmp(n2);
      for (u64 p = 0; p < n2; ++p) tmp[p] = ts->Wo[p + n2 * l] * (this->S[p + n2 * c] * x[p]);
      ts->G->forward(tmp.data(), out.data() + n1 * u);
    });
    for (u64 c = 0; c < nc; ++c) {
      C* yc = y + n1 * c;
      std::fill(yc, yc + n1, C(0, 0));
      for (u64 l = 0; l < L; ++l)
        for (u64 m = 0; m < n1; ++m) yc[m] += out[n1 * (c * L + l) + m] * ts->AA[m + n1 * l];
    }
  }
  void adjoint(const C* d, C* x) const override {
    auto* ts = dynamic_cast<const pgo::TimeSegOp<T>*>(this->G);
    if (!ts || g_threads <= 1) return pgo::SenseOp<T>::adjoint(d, x);
    const u64 n1 = this->n1, n2 = this->n2, L = ts->L, nc = this->nc;
    std::vector<C> img(n2 * L * nc);
    parallel_for(nc * L, [&](u64 u) {
      const u64 c = u / L, l = u % L;
      std::vector<C> tmp(n1);
      const C* dc = d + n1 * c;
      for (u64 m = 0; m < n1; ++m) tmp[m] = std::conj(ts->AA[m + n1 * l]) * dc[m];
      ts->G->adjoint(tmp.data(), img.data() + n2 * u);
    });
    std::fill(x, x + n2, C(0, 0));
    std::vector<C> xc(n2);
    for (u64 c = 0; c < nc; ++c) {
      std::fill(xc.begin(), xc.end(), C(0, 0));
      for (u64 l = 0; l < L; ++l)
        for (u64 p = 0; p < n2; ++p) xc[p] += img[n2 * (c * L + l) + p] * ts->WoH[p + n2 * l];
      for (u64 p = 0; p < n2; ++p) x[p] += xc[p] * std::conj(this->S[p + n2 * c]);
    }
  }
};

// pcSenseTimeSeg with its (coil, shot, segment) Gnufft calls spread over
// threads.  Per-element arithmetic and summation order equal the serial
// loops of PcSenseTimeSegOp and TimeSegOp (pcSenseTimeSeg.cpp:127-171,
// TimeSegmentation.cpp:252-324).
template <typename T>
struct PcSenseTsParallel : pgo::PcSenseTimeSegOp<T> {
  using C = std::complex<T>;
  using pgo::PcSenseTimeSegOp<T>::PcSenseTimeSegOp;
  void forward(const C* x, C* y) const override {
    if (g_threads <= 1) return pgo::PcSenseTimeSegOp<T>::forward(x, y);
    const u64 Ni = this->Ni, Nd = this->Nd, Ns = this->Ns, Nc = this->Nc, L = (u64)this->A[0]->L;
    std::vector<C> out(Nd * L * Ns * Nc);
    parallel_for(Nc * Ns * L, [&](u64 u) {
      const u64 l = u % L, cs = u / L, s = cs % Ns;   // cs = s + c*Ns
      const auto* ts = this->A[s].get();
      const C* m = this->M.data() + Ni * cs;
      std::vector<C> tmp(Ni);
      for (u64 p = 0; p < Ni; ++p) tmp[p] = ts->Wo[p + Ni * l] * (x[p] * m[p]);
      ts->G->forward(tmp.data(), out.data() + Nd * u);
    });
    for (u64 cs = 0; cs < Nc * Ns; ++cs) {
      const auto* ts = this->A[cs % Ns].get();
      C* yc = y + Nd * cs;
      std::fill(yc, yc + Nd, C(0, 0));
      for (u64 l = 0; l < L; ++l)
        for (u64 q = 0; q < Nd; ++q) yc[q] += out[Nd * (cs * L + l) + q] * ts->AA[q + Nd * l];
    }
  }
  void adjoint(const C* d, C* x) const override {
    if (g_threads <= 1) return pgo::PcSenseTimeSegOp<T>::adjoint(d, x);
    const u64 Ni = this->Ni, Nd = this->Nd, Ns = this->Ns, Nc = this->Nc, L = (u64)this->A[0]->L;
    std::vector<C> img(Ni * L * Ns * Nc);
    parallel_for(Nc * Ns * L, [&](u64 u) {
      const u64 l = u % L, cs = u / L, s = cs % Ns;
      const auto* ts = this->A[s].get();
      const C* dc = d + Nd * cs;
      std::vector<C> tmp(Nd);
      for (u64 q = 0; q < Nd; ++q) tmp[q] = std::conj(ts->AA[q + Nd * l]) * dc[q];
      ts->G->adjoint(tmp.data(), img.data() + Ni * u);
    });
    std::fill(x, x + Ni, C(0, 0));
    std::vector<C> xs(Ni);
    for (u64 cs = 0; cs < Nc * Ns; ++cs) {
      const auto* ts = this->A[cs % Ns].get();
      std::fill(xs.begin(), xs.end(), C(0, 0));
      for (u64 l = 0; l < L; ++l)
        for (u64 p = 0; p < Ni; ++p) xs[p] += img[Ni * (cs * L + l) + p] * ts->WoH[p + Ni * l];
      const C* m = this->Mc.data() + Ni * cs;
      for (u64 p = 0; p < Ni; ++p) x[p] += m[p] * xs[p];
    }
  }
};

struct Handle {
  int prec;
  std::unique_ptr<pgo::Op<float>> f;
  std::unique_ptr<pgo::Op<double>> d;
};

template <typename T>
std::vector<T> widen(const float* p, u64 n) {
  std::vector<T> v(n);
  for (u64 i = 0; i < n; ++i) v[i] = (T)p[i];
  return v;
}

template <typename T>
pgo::Op<T>* get(Handle* h);
template <>
pgo::Op<float>* get<float>(Handle* h) { return h->f.get(); }
template <>
pgo::Op<double>* get<double>(Handle* h) { return h->d.get(); }

template <typename T>
void set(Handle* h, pgo::Op<T>* op);
template <>
void set<float>(Handle* h, pgo::Op<float>* op) { h->f.reset(op); }
template <>
void set<double>(Handle* h, pgo::Op<double>* op) { h->d.reset(op); }

// An FP64 view of a float operator: the input is rounded to float, the float
// operator applied and its output widened.  Solving over it in FP64 leaves
// the operator's FP32 rounding as the only FP32 step, which separates the
// operator's share of a float solve's error from the solver's.
struct WidenedOp : pgo::Op<double> {
  const pgo::Op<float>* f = nullptr;
  void forward(const std::complex<double>* x, std::complex<double>* y) const override {
    std::vector<std::complex<float>> xf(n2), yf(n1);
    for (u64 i = 0; i < n2; ++i) xf[i] = std::complex<float>((float)x[i].real(), (float)x[i].imag());
    f->forward(xf.data(), yf.data());
    for (u64 i = 0; i < n1; ++i) y[i] = std::complex<double>(yf[i].real(), yf[i].imag());
  }
  void adjoint(const std::complex<double>* y, std::complex<double>* x) const override {
    std::vector<std::complex<float>> yf(n1), xf(n2);
    for (u64 i = 0; i < n1; ++i) yf[i] = std::complex<float>((float)y[i].real(), (float)y[i].imag());
    f->adjoint(yf.data(), xf.data());
    for (u64 i = 0; i < n2; ++i) x[i] = std::complex<double>(xf[i].real(), xf[i].imag());
  }
};

template <typename F>
void* guard(F fn) {
  try {
    return fn();
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

}  // namespace

namespace {
template <typename T>
pgo::LowRankPenalty<T> lowrank_penalty(const pgo::Penalty<T>& R, u64 rank, const float* v) {
  pgo::LowRankPenalty<T> P;
  P.R = &R;
  P.K = rank;
  P.v.resize(rank * rank);
  for (u64 i = 0; i < rank * rank; ++i) P.v[i] = std::complex<T>((T)v[2 * i], (T)v[2 * i + 1]);
  return P;
}
}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

int orc_use_reference(const char* so_path) {
  if (!so_path) { g_use_ref = false; return 0; }
  void* h = dlopen(so_path, RTLD_NOW | RTLD_LOCAL);
  if (!h) { g_err = dlerror(); return -1; }
  auto& kf = pgo::ref_kernels<float>();
  auto& kd = pgo::ref_kernels<double>();
  kf.fd = (decltype(kf.fd))dlsym(h, "pgref_fd_f");
  kf.fh = (decltype(kf.fh))dlsym(h, "pgref_fh_f");
  kf.ft = (decltype(kf.ft))dlsym(h, "pgref_ft_f");
  kf.ift = (decltype(kf.ift))dlsym(h, "pgref_ift_f");
  kd.fd = (decltype(kd.fd))dlsym(h, "pgref_fd_d");
  kd.fh = (decltype(kd.fh))dlsym(h, "pgref_fh_d");
  kd.ft = (decltype(kd.ft))dlsym(h, "pgref_ft_d");
  kd.ift = (decltype(kd.ift))dlsym(h, "pgref_ift_d");
  kf.ftg = (decltype(kf.ftg))dlsym(h, "pgref_ftg_f");
  kf.iftg = (decltype(kf.iftg))dlsym(h, "pgref_iftg_f");
  kf.ifwd = (decltype(kf.ifwd))dlsym(h, "pgref_ifwd_f");
  kf.iadj = (decltype(kf.iadj))dlsym(h, "pgref_iadj_f");
  kd.ifwd = (decltype(kd.ifwd))dlsym(h, "pgref_ifwd_d");
  kd.iadj = (decltype(kd.iadj))dlsym(h, "pgref_iadj_d");
  if (!kf.fd || !kf.fh || !kf.ft || !kf.ift || !kd.fd || !kd.fh || !kd.ft || !kd.ift || !kf.ifwd || !kf.iadj ||
      !kd.ifwd || !kd.iadj || !kf.ftg || !kf.iftg) {
    g_err = "libpgref.so lacks an expected symbol";
    return -1;
  }
  g_use_ref = true;
  return 0;
}

// Kaiser-Bessel LUT and beta as Gnufft builds them (precision 0 -> float out, else double out).
int orc_kb_lut(int prec, float gridos, void* out, u64 cap, double* beta_out) {
  if (prec == 0) {
    float beta = pgo::kb_beta<float>(gridos, 4.0f);
    auto lut = pgo::kb_lut<float>(beta, 4.0f);
    if (lut.size() > cap) return -1;
    std::memcpy(out, lut.data(), lut.size() * sizeof(float));
    *beta_out = beta;
    return (int)lut.size();
  }
  double beta = pgo::kb_beta<double>(gridos, 4.0);
  auto lut = pgo::kb_lut<double>(beta, 4.0);
  if (lut.size() > cap) return -1;
  std::memcpy(out, lut.data(), lut.size() * sizeof(double));
  *beta_out = beta;
  return (int)lut.size();
}

void* orc_gnufft_new(int prec, u64 M, float gridos, u64 nx, u64 ny, u64 nz, const float* kx, const float* ky,
                     const float* kz) {
  return guard([&]() -> void* {
    auto* h = new Handle;
    h->prec = prec;
    if (prec == 0) {
      auto* op = new pgo::GnufftOp<float>(M, gridos, (int)nx, (int)ny, (int)nz, kx, ky, kz);
      op->use_ref = g_use_ref;
      h->f.reset(op);
    } else {
      auto a = widen<double>(kx, M), b = widen<double>(ky, M), c = widen<double>(kz, M);
      auto* op = new pgo::GnufftOp<double>(M, gridos, (int)nx, (int)ny, (int)nz, a.data(), b.data(), c.data());
      if (prec == 3)
        op->use_float_taps();
      else
        op->use_ref = g_use_ref;
      h->d.reset(op);
    }
    return h;
  });
}

void* orc_gdft_new(int prec, u64 nk, u64 ni, const float* kx, const float* ky, const float* kz, const float* ix,
                   const float* iy, const float* iz, const float* fm, const float* t) {
  return guard([&]() -> void* {
    auto* h = new Handle;
    h->prec = prec;
    if (prec == 0) {
      auto* op = new pgo::GdftOp<float>(nk, ni, kx, ky, kz, ix, iy, iz, fm, t);
      op->use_ref = g_use_ref;
      h->f.reset(op);
    } else {
      auto a = widen<double>(kx, nk), b = widen<double>(ky, nk), c = widen<double>(kz, nk);
      auto d = widen<double>(ix, ni), e = widen<double>(iy, ni), f = widen<double>(iz, ni);
      auto g = widen<double>(fm, ni), tt = widen<double>(t, nk);
      auto* op = new pgo::GdftOp<double>(nk, ni, a.data(), b.data(), c.data(), d.data(), e.data(), f.data(),
                                         g.data(), tt.data());
      op->exact64 = (prec == 2);
      op->use_ref = g_use_ref;
      h->d.reset(op);
    }
    return h;
  });
}

// tables64: min-max / histogram tables built in double and rounded (float handles only)
// prec: 0 float, 1 double (reference formula), 2 double with the FP64 DFT
void* orc_gdftr2_new(int prec, u64 nk, u64 ni, const float* kx, const float* ky, const float* kz, const float* ix,
                     const float* iy, const float* iz, const float* fm, const float* t, u64 nx, u64 ny, u64 nz) {
  return guard([&]() -> void* {
    auto* h = new Handle;
    h->prec = prec;
    if (prec == 0) {
      auto* op = new pgo::GdftR2Op<float>(nk, ni, kx, ky, kz, ix, iy, iz, fm, t, (int)nx, (int)ny, (int)nz);
      op->use_ref = g_use_ref;
      h->f.reset(op);
    } else {
      auto a = widen<double>(kx, nk), b = widen<double>(ky, nk), c = widen<double>(kz, nk);
      auto d = widen<double>(ix, ni), e = widen<double>(iy, ni), f = widen<double>(iz, ni);
      auto g = widen<double>(fm, ni), tt = widen<double>(t, nk);
      auto* op = new pgo::GdftR2Op<double>(nk, ni, a.data(), b.data(), c.data(), d.data(), e.data(), f.data(),
                                           g.data(), tt.data(), (int)nx, (int)ny, (int)nz);
      op->exact64 = (prec == 2);
      h->d.reset(op);
    }
    return h;
  });
}

void* orc_timeseg_new(void* G, const float* fieldmap, const float* tvec, u64 n1, u64 n2, u64 L, u64 type,
                      u64 shots, int tables64) {
  return guard([&]() -> void* {
    Handle* g = (Handle*)G;
    auto* h = new Handle;
    h->prec = g->prec;
    if (g->prec == 0) {
      h->f.reset(new pgo::TimeSegOp<float>(g->f.get(), fieldmap, tvec, n1, n2, L, type, shots, tables64 != 0));
    } else {
      auto fm = widen<double>(fieldmap, n2), tv = widen<double>(tvec, n1);
      h->d.reset(new pgo::TimeSegOp<double>(g->d.get(), fm.data(), tv.data(), n1, n2, L, type, shots));
    }
    return h;
  });
}

// smap: complex64 interleaved n2*nc (coil-major)
void* orc_sense_new(void* G, const float* smap, u64 n1, u64 n2, u64 nc) {
  return guard([&]() -> void* {
    Handle* g = (Handle*)G;
    auto* h = new Handle;
    h->prec = g->prec;
    const std::complex<float>* s = reinterpret_cast<const std::complex<float>*>(smap);
    if (g->prec == 0) {
      h->f.reset(new SenseParallel<float>(g->f.get(), s, n1, n2, nc));
    } else {
      std::vector<std::complex<double>> sd(n2 * nc);
      for (u64 i = 0; i < n2 * nc; ++i) sd[i] = std::complex<double>(s[i].real(), s[i].imag());
      h->d.reset(new SenseParallel<double>(g->d.get(), sd.data(), n1, n2, nc));
    }
    return h;
  });
}

void* orc_pcsense_ts_new(int prec, const float* kx, const float* ky, const float* kz, u64 nk, u64 nx, u64 ny,
                         u64 nz, u64 nc, const float* t, u64 L, u64 type, const float* smap, const float* fmap,
                         const float* pmap, u64 npmap) {
  return guard([&]() -> void* {
    auto* h = new Handle;
    h->prec = prec;
    const u64 ni = nx * ny * nz;
    const std::complex<float>* s = reinterpret_cast<const std::complex<float>*>(smap);
    if (prec == 0) {
      h->f.reset(new PcSenseTsParallel<float>(kx, ky, kz, nk, (int)nx, (int)ny, (int)nz, nc, t, L, type, s,
                                              fmap, pmap, npmap, g_use_ref));
    } else {
      auto a = widen<double>(kx, nk), b = widen<double>(ky, nk), c = widen<double>(kz, nk);
      auto tt = widen<double>(t, nk), fm = widen<double>(fmap, ni), pm = widen<double>(pmap, npmap);
      std::vector<std::complex<double>> sd(ni * nc);
      for (u64 i = 0; i < ni * nc; ++i) sd[i] = std::complex<double>(s[i].real(), s[i].imag());
      auto* op = new PcSenseTsParallel<double>(a.data(), b.data(), c.data(), nk, (int)nx, (int)ny, (int)nz,
                                               nc, tt.data(), L, type, sd.data(), fm.data(), pm.data(), npmap,
                                               g_use_ref && prec != 3);
      if (prec == 3)
        for (auto& g : op->G) g->use_float_taps();
      h->d.reset(op);
    }
    return h;
  });
}

// prec: 0 float, 1 double (reference DFT formula), 2 double with the FP64 DFT
void* orc_pcsense_new(int prec, const float* kx, const float* ky, const float* kz, u64 nk, u64 nx, u64 ny, u64 nz,
                      u64 nc, const float* t, const float* smap, const float* fmap, const float* pmap, u64 npmap) {
  return guard([&]() -> void* {
    auto* h = new Handle;
    h->prec = prec;
    const u64 ni = nx * ny * nz;
    const std::complex<float>* s = reinterpret_cast<const std::complex<float>*>(smap);
    if (prec == 0) {
      h->f.reset(new pgo::PcSenseOp<float>(kx, ky, kz, nk, (int)nx, (int)ny, (int)nz, nc, t, s, fmap, pmap, npmap,
                                           g_use_ref, false));
    } else {
      auto a = widen<double>(kx, nk), b = widen<double>(ky, nk), c = widen<double>(kz, nk);
      auto tt = widen<double>(t, nk), fm = widen<double>(fmap, ni), pm = widen<double>(pmap, npmap);
      std::vector<std::complex<double>> sd(ni * nc);
      for (u64 i = 0; i < ni * nc; ++i) sd[i] = std::complex<double>(s[i].real(), s[i].imag());
      h->d.reset(new pgo::PcSenseOp<double>(a.data(), b.data(), c.data(), nk, (int)nx, (int)ny, (int)nz, nc,
                                            tt.data(), sd.data(), fm.data(), pm.data(), npmap, g_use_ref, prec == 2));
    }
    return h;
  });
}

void orc_free(void* h) { delete (Handle*)h; }

u64 orc_data_len(void* h) {
  Handle* x = (Handle*)h;
  return x->prec == 0 ? pgo::op_data_len(*x->f) : pgo::op_data_len(*x->d);
}
u64 orc_image_len(void* h) {
  Handle* x = (Handle*)h;
  return x->prec == 0 ? pgo::op_image_len(*x->f) : pgo::op_image_len(*x->d);
}

int orc_forward(void* h, const void* x, void* y) {
  Handle* o = (Handle*)h;
  if (o->prec == 0)
    o->f->forward((const std::complex<float>*)x, (std::complex<float>*)y);
  else
    o->d->forward((const std::complex<double>*)x, (std::complex<double>*)y);
  return 0;
}
int orc_adjoint(void* h, const void* y, void* x) {
  Handle* o = (Handle*)h;
  if (o->prec == 0)
    o->f->adjoint((const std::complex<float>*)y, (std::complex<float>*)x);
  else
    o->d->adjoint((const std::complex<double>*)y, (std::complex<double>*)x);
  return 0;
}

// Spatial interpolation of a Gnufft handle (grid in the reference's layout).
u64 orc_gnufft_grid_len(void* h) {
  Handle* o = (Handle*)h;
  if (o->prec == 0) return dynamic_cast<pgo::GnufftOp<float>&>(*o->f).g.ngrid();
  return dynamic_cast<pgo::GnufftOp<double>&>(*o->d).g.ngrid();
}
int orc_gnufft_interp_fwd(void* h, const void* grid, void* y) {
  Handle* o = (Handle*)h;
  if (o->prec == 0)
    dynamic_cast<pgo::GnufftOp<float>&>(*o->f).forward_interp((const std::complex<float>*)grid,
                                                               (std::complex<float>*)y);
  else
    dynamic_cast<pgo::GnufftOp<double>&>(*o->d).forward_interp((const std::complex<double>*)grid,
                                                                (std::complex<double>*)y);
  return 0;
}
int orc_gnufft_interp_adj(void* h, const void* d, void* grid) {
  Handle* o = (Handle*)h;
  if (o->prec == 0)
    dynamic_cast<pgo::GnufftOp<float>&>(*o->f).adjoint_interp((const std::complex<float>*)d,
                                                               (std::complex<float>*)grid);
  else
    dynamic_cast<pgo::GnufftOp<double>&>(*o->d).adjoint_interp((const std::complex<double>*)d,
                                                                (std::complex<double>*)grid);
  return 0;
}

// calc3DDensityCompensation; out: n floats (prec 0) or doubles.
int orc_density_compensation(int prec, const float* kx, const float* ky, const float* kz, u64 n, u64 ninplane,
                             u64 nz, void* out) {
  if (prec == 0) {
    auto v = pgo::density_compensation<float>(kx, ky, kz, n, (int)ninplane, (int)nz, g_use_ref);
    std::memcpy(out, v.data(), n * sizeof(float));
  } else {
    auto a = widen<double>(kx, n), b = widen<double>(ky, n), c = widen<double>(kz, n);
    auto v = pgo::density_compensation<double>(a.data(), b.data(), c.data(), n, (int)ninplane, (int)nz, g_use_ref);
    std::memcpy(out, v.data(), n * sizeof(double));
  }
  return 0;
}

// reconSolve-style PWLS-PCG (solve_pwls_pcg.hpp:48-167).  W: real vector in
// the operator's precision (nullptr -> ones, as reconSolve.h:73-74).
int orc_pcg(void* h, const void* x0, const void* W, const void* y, int kind, u64 nx, u64 ny, u64 nz, double beta,
            double delta, u64 dims2pen, u64 niter, void* xout) {
  Handle* o = (Handle*)h;
  auto run = [&](auto* op, auto tag) -> int {
    using T = decltype(tag);
    pgo::Penalty<T> R;
    R.kind = kind; R.Nx = nx; R.Ny = ny; R.Nz = nz; R.beta = (T)beta; R.delta = (T)delta; R.dims2pen = dims2pen;
    const u64 nd = pgo::op_data_len(*op), ni = pgo::op_image_len(*op);
    std::vector<T> w(nd, (T)1);
    if (W) std::memcpy(w.data(), W, sizeof(T) * nd);
    std::vector<std::complex<T>> xi(ni, std::complex<T>(0, 0));
    if (x0) std::memcpy(xi.data(), x0, sizeof(std::complex<T>) * ni);
    return pgo::pwls_pcg<T>(*op, xi.data(), w.data(), (const std::complex<T>*)y, R, niter,
                            (std::complex<T>*)xout);
  };
  if (o->prec == 0) return run(o->f.get(), float());
  return run(o->d.get(), double());
}

// PWLS-PCG in FP64 (vectors, inner products, steps) over a float (precision 0)
// operator.  y and xout are complex128; W, if given, double.
int orc_pcg_fp64_over_f32(void* h, const void* W, const void* y, int kind, u64 nx, u64 ny, u64 nz, double beta,
                          double delta, u64 dims2pen, u64 niter, void* xout) {
  Handle* o = (Handle*)h;
  if (o->prec != 0) { g_err = "orc_pcg_fp64_over_f32 needs a float operator"; return -1; }
  WidenedOp A;
  A.f = o->f.get();
  A.n1 = pgo::op_data_len(*A.f);
  A.n2 = pgo::op_image_len(*A.f);
  pgo::Penalty<double> R;
  R.kind = kind; R.Nx = nx; R.Ny = ny; R.Nz = nz; R.beta = beta; R.delta = delta; R.dims2pen = dims2pen;
  std::vector<double> w(A.n1, 1.0);
  if (W) std::memcpy(w.data(), W, sizeof(double) * A.n1);
  std::vector<std::complex<double>> xi(A.n2, std::complex<double>(0, 0));
  return pgo::pwls_pcg<double>(A, xi.data(), w.data(), (const std::complex<double>*)y, R, niter,
                               (std::complex<double>*)xout);
}

// LRobj over oracle operators (lowRank/LRobj.cpp:27-68); the operators are
// borrowed and must outlive it.  v: rank x n_img complex float, column-major.
void* orc_lowrank_new(u64 n_image, u64 n_data, u64 rank, u64 n_img, const float* v, void* const* ops) {
  return guard([&]() -> void* {
    const int prec = ((Handle*)ops[0])->prec;
    auto* h = new Handle;
    h->prec = prec;
    auto make = [&](auto tag) {
      using T = decltype(tag);
      std::vector<std::complex<T>> vb(rank * n_img);
      for (u64 i = 0; i < rank * n_img; ++i) vb[i] = std::complex<T>((T)v[2 * i], (T)v[2 * i + 1]);
      std::vector<const pgo::Op<T>*> A;
      for (u64 i = 0; i < n_img; ++i) A.push_back(get<T>((Handle*)ops[i]));
      set<T>(h, new pgo::LowRankOp<T>(n_image, n_data, rank, n_img, vb.data(), A));
    };
    if (prec == 0) make(float()); else make(double());
    return h;
  });
}

// solve_pwls_pcg<T1, LRobj, R_lowRank> (lowRank/oscillateRecon.cpp:260-265
// composes it); R_lowRank's basis is rank x rank (rank == number of images).
int orc_pcg_lowrank(void* h, const void* x0, const void* W, const void* y, int kind, u64 nx, u64 ny, u64 nz,
                    double beta, double delta, u64 dims2pen, u64 rank, const float* v, u64 niter, void* xout) {
  Handle* o = (Handle*)h;
  auto run = [&](auto* op, auto tag) -> int {
    using T = decltype(tag);
    pgo::Penalty<T> R;
    R.kind = kind; R.Nx = nx; R.Ny = ny; R.Nz = nz; R.beta = (T)beta; R.delta = (T)delta; R.dims2pen = dims2pen;
    const pgo::LowRankPenalty<T> P = lowrank_penalty(R, rank, v);
    const u64 nd = pgo::op_data_len(*op), ni = pgo::op_image_len(*op);
    std::vector<T> w(nd, (T)1);
    if (W) std::memcpy(w.data(), W, sizeof(T) * nd);
    std::vector<std::complex<T>> xi(ni, std::complex<T>(0, 0));
    if (x0) std::memcpy(xi.data(), x0, sizeof(std::complex<T>) * ni);
    return pgo::pwls_pcg<T>(*op, xi.data(), w.data(), (const std::complex<T>*)y, P, niter,
                            (std::complex<T>*)xout);
  };
  if (o->prec == 0) return run(o->f.get(), float());
  return run(o->d.get(), double());
}

// R_lowRank pieces for unit tests (lowRank/R_lowRank.cpp:50-87).
int orc_lowrank_gradient(int prec, int kind, u64 nx, u64 ny, u64 nz, double beta, double delta, u64 dims2pen,
                         u64 rank, const float* v, const void* x, void* g) {
  auto run = [&](auto tag) {
    using T = decltype(tag);
    pgo::Penalty<T> R;
    R.kind = kind; R.Nx = nx; R.Ny = ny; R.Nz = nz; R.beta = (T)beta; R.delta = (T)delta; R.dims2pen = dims2pen;
    lowrank_penalty(R, rank, v).Gradient((const std::complex<T>*)x, (std::complex<T>*)g);
  };
  if (prec == 0) run(float()); else run(double());
  return 0;
}
int orc_lowrank_denom(int prec, int kind, u64 nx, u64 ny, u64 nz, double beta, double delta, u64 dims2pen,
                      u64 rank, const float* v, const void* ddir, const void* x, double* out2) {
  auto run = [&](auto tag) {
    using T = decltype(tag);
    pgo::Penalty<T> R;
    R.kind = kind; R.Nx = nx; R.Ny = ny; R.Nz = nz; R.beta = (T)beta; R.delta = (T)delta; R.dims2pen = dims2pen;
    auto d = lowrank_penalty(R, rank, v).Denom((const std::complex<T>*)ddir, (const std::complex<T>*)x);
    out2[0] = d.real(); out2[1] = d.imag();
  };
  if (prec == 0) run(float()); else run(double());
  return 0;
}

// Regularizer pieces for unit tests: Gradient and Denom (Robject.cpp:143-193).
int orc_penalty_gradient(int prec, int kind, u64 nx, u64 ny, u64 nz, double beta, double delta, u64 dims2pen,
                         const void* x, void* g) {
  auto run = [&](auto tag) {
    using T = decltype(tag);
    pgo::Penalty<T> R;
    R.kind = kind; R.Nx = nx; R.Ny = ny; R.Nz = nz; R.beta = (T)beta; R.delta = (T)delta; R.dims2pen = dims2pen;
    R.Gradient((const std::complex<T>*)x, (std::complex<T>*)g);
  };
  if (prec == 0) run(float()); else run(double());
  return 0;
}
int orc_penalty_denom(int prec, int kind, u64 nx, u64 ny, u64 nz, double beta, double delta, u64 dims2pen,
                      const void* ddir, const void* x, double* out2) {
  auto run = [&](auto tag) {
    using T = decltype(tag);
    pgo::Penalty<T> R;
    R.kind = kind; R.Nx = nx; R.Ny = ny; R.Nz = nz; R.beta = (T)beta; R.delta = (T)delta; R.dims2pen = dims2pen;
    auto v = R.Denom((const std::complex<T>*)ddir, (const std::complex<T>*)x);
    out2[0] = v.real(); out2[1] = v.imag();
  };
  if (prec == 0) run(float()); else run(double());
  return 0;
}

// Time-segmentation tables (AA n1 x L, Wo/WoH n2 x (L+1)) for unit tests.
int orc_timeseg_tables(void* h, void* AA, void* Wo, void* WoH, double* tau_tmin) {
  Handle* o = (Handle*)h;
  if (o->prec == 0) {
    auto* ts = dynamic_cast<pgo::TimeSegOp<float>*>(o->f.get());
    if (!ts) return -1;
    if (AA) std::memcpy(AA, ts->AA.data(), sizeof(ts->AA[0]) * ts->n1 * ts->L);
    if (Wo) std::memcpy(Wo, ts->Wo.data(), sizeof(ts->Wo[0]) * ts->Wo.size());
    if (WoH) std::memcpy(WoH, ts->WoH.data(), sizeof(ts->WoH[0]) * ts->WoH.size());
    tau_tmin[0] = ts->tau; tau_tmin[1] = ts->tmin;
    return ts->L;
  }
  auto* ts = dynamic_cast<pgo::TimeSegOp<double>*>(o->d.get());
  if (!ts) return -1;
  if (AA) std::memcpy(AA, ts->AA.data(), sizeof(ts->AA[0]) * ts->n1 * ts->L);
  if (Wo) std::memcpy(Wo, ts->Wo.data(), sizeof(ts->Wo[0]) * ts->Wo.size());
  if (WoH) std::memcpy(WoH, ts->WoH.data(), sizeof(ts->WoH[0]) * ts->WoH.size());
  tau_tmin[0] = ts->tau; tau_tmin[1] = ts->tmin;
  return ts->L;
}

// Raw N-d FFT (for validating the project FFT against numpy).
int orc_fft(int prec, void* data, const u64* dims, int rank, int sign) {
  std::vector<std::size_t> d(dims, dims + rank);
  if (prec == 0)
    pgo::fft_nd<float>((std::complex<float>*)data, d.data(), rank, sign);
  else
    pgo::fft_nd<double>((std::complex<double>*)data, d.data(), rank, sign);
  return 0;
}

}  // extern "C"
