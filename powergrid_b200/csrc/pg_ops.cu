// Operators and their C ABI.  A composite recognises the operator under it
// and runs the whole composition as one batched device pipeline:
//   SENSE<TimeSegmentation<Gnufft>>  -> one NUFFT pass over coils x segments
//   SENSE<Gnufft>, TimeSegmentation<Gnufft>, Gnufft -> the same pass, fewer factors
//   SENSE<Gdft>, Gdft                -> one coil-batched DFT pass
// Any other nesting falls back to composing the inner operator's device
// calls with element-wise kernels (still on the GPU).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "pg_ops.cuh"

namespace pg {

// ---- element-wise kernels for the generic composition path ----------------
__global__ void k_cmul(uint64_t n, const float2* __restrict__ a, const float2* __restrict__ b, int conj_a,
                       float2* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 av = conj_a ? cconj(a[i]) : a[i];
  out[i] = cmul(av, b[i]);
}
// out (+)= a (.) b  (conj_b selects conj(b))
__global__ void k_cmul_acc(uint64_t n, const float2* __restrict__ a, const float2* __restrict__ b, int conj_b,
                           int accumulate, float2* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 bv = conj_b ? cconj(b[i]) : b[i];
  const float2 v = cmul(a[i], bv);
  out[i] = accumulate ? cadd(out[i], v) : v;
}

// ---- time-segmentation tables ---------------------------------------------
pg_status build_ts_tables(const float* field_map, const float* tvec, uint64_t n1, uint64_t n2, uint64_t Lin,
                          uint64_t interptype, uint64_t shots, TsTables* out) {
  TsTables& T = *out;
  if (n1 == 0 || n2 == 0) return set_error(PG_INVALID_ARG, "TimeSegmentation: empty sizes");
  if (shots == 0 || n1 % shots) return set_error(PG_INVALID_ARG, "TimeSegmentation: n1 not divisible by shots");
  for (uint64_t m = 0; m < n1; ++m)
    if (!std::isfinite(tvec[m])) return set_error(PG_INVALID_ARG, "TimeSegmentation: non-finite time at %llu",
                                                  (unsigned long long)m);
  for (uint64_t p = 0; p < n2; ++p)
    if (!std::isfinite(field_map[p])) return set_error(PG_INVALID_ARG, "TimeSegmentation: non-finite field map");
  // TimeSegmentation.cpp:46-50: L in {0,1} means no segmentation.
  int L = (Lin == 0 || Lin == 1) ? 1 : (int)Lin;
  if (L > 64) return set_error(PG_INVALID_ARG, "TimeSegmentation: L=%d exceeds 64", L);
  if (L > 1 && (interptype < 1 || interptype > 3))
    return set_error(PG_INVALID_ARG, "TimeSegmentation: interptype %llu (1 Hanning, 2 min-max, 3 histogram)",
                     (unsigned long long)interptype);
  std::vector<float> tv(tvec, tvec + n1);
  float mn = tv[0], mx = tv[0];
  for (float v : tv) { mn = std::min(mn, v); mx = std::max(mx, v); }
  T.tmin = mn;
  const float rangt = mx - T.tmin;
  T.tau = (rangt + std::numeric_limits<double>::epsilon()) / L;  // :66-68 (datum::eps is double eps)
  for (auto& v : tv) v = v - T.tmin;
  T.L = L;
  if (L <= 1) {
    T.L = 1; T.tau = 0; T.K = 1;
    return PG_OK;
  }
  const uint64_t none = n1 / shots;
  const double kPi = 3.141592653589793238462643383279502884;  // arma datum::pi
  std::vector<float2> one(none * L);
  if (interptype == 1) {
    // Hanning interpolator (:83-92), repeated over shots.
    for (unsigned int l = 0; l < (unsigned)L; ++l)
      for (unsigned int m = 0; m < none; ++m) {
        float v = 0.f;
        if ((std::abs(tv[m] - ((l) * T.tau))) <= T.tau)
          v = (float)(0.5 + 0.5 * std::cos((kPi) * (tv[m] - ((l) * T.tau)) / T.tau));
        one[m + none * l] = make_float2(v, 0.f);
      }
  } else {
    // min-max (:94-156) or its histogram approximation (:157-211), over one shot's times
    const std::vector<float> t1(tv.begin(), tv.begin() + none);
    if (interptype == 2)
      PG_TRY(ts_aa_minmax(field_map, n2, t1, L, T.tau, &one));
    else
      PG_TRY(ts_aa_histogram(field_map, n2, t1, L, T.tau, &one));
  }
  T.AA.resize(n1 * L);
  for (int l = 0; l < L; ++l)
    for (uint64_t m = 0; m < n1; ++m) T.AA[m + n1 * l] = one[(m % none) + none * l];
  // Segment window per sample: the span of nonzero AA entries.
  std::vector<int> first(n1, 0), last(n1, -1);
  int K = 1;
  for (uint64_t m = 0; m < n1; ++m) {
    for (int l = 0; l < L; ++l) {
      const float2 a = T.AA[m + n1 * l];
      if (a.x != 0.f || a.y != 0.f) {
        if (last[m] < 0) first[m] = l;
        last[m] = l;
      }
    }
    if (last[m] >= 0) K = std::max(K, last[m] - first[m] + 1);
  }
  T.K = K;
  T.l0.resize(n1);
  T.aa_win.resize(n1 * (uint64_t)K);
  for (uint64_t m = 0; m < n1; ++m) {
    const int s = std::min(first[m], L - K);
    T.l0[m] = s;
    for (int q = 0; q < K; ++q) T.aa_win[m * K + q] = T.AA[m + n1 * (s + q)];
  }
  return PG_OK;
}

// Wo / WoH (TimeSegmentation.cpp:213-218): exp(-/+ i * fieldMap * (l*tau + T_min)),
// l < L, evaluated on the device (the host loop over N x L sincos dominated
// operator set-up).  sincosf is the accurate CUDA routine, not the fast
// intrinsic; the argument is formed with the reference's float rounding.
__global__ void k_ts_phases(uint64_t n2, int L, float tau, float tmin, const float* __restrict__ fm,
                            float2* __restrict__ Wo, float2* __restrict__ WoH) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n2 * (uint64_t)L) return;
  const unsigned int l = (unsigned int)(i / n2);
  const uint64_t p = i % n2;
  const float sft = __fadd_rn(__fmul_rn((float)l, tau), tmin);
  const float v = __fmul_rn(fm[p], sft);
  float sn, c;
  sincosf(v, &sn, &c);
  Wo[i] = make_float2(c, -sn);
  WoH[i] = make_float2(c, sn);
}

pg_status build_ts_phases(const TsTables& T, const float* field_map, uint64_t n2, DevBuf<float2>* Wo,
                          DevBuf<float2>* WoH, cudaStream_t s) {
  DevBuf<float> fm;
  PG_TRY(fm.upload(field_map, n2, s));
  PG_TRY(Wo->alloc(n2 * (uint64_t)T.L));
  PG_TRY(WoH->alloc(n2 * (uint64_t)T.L));
  PG_LAUNCH(k_ts_phases, ceil_div(n2 * (uint64_t)T.L, 256), 256, 0, s, n2, T.L, T.tau, T.tmin, fm.p, Wo->p, WoH->p);
  PG_CUDA(cudaStreamSynchronize(s));  // fm is released on return
  return PG_OK;
}

// ---- Gnufft ------------------------------------------------------------------
static pg_status interp_only() {
  return set_error(PG_INVALID_ARG, "Gnufft: operator application needs gridos = 2 (other factors: spatial "
                                   "interpolation only)");
}

pg_status GnufftOp::forward(const float2* x, float2* y, cudaStream_t s) {
  if (!plan) return interp_only();
  NufftBatch b;
  b.C = 1;
  b.data_stride = plan->M;
  return nufft_forward(plan.get(), b, x, y, s);
}
pg_status GnufftOp::adjoint(const float2* y, float2* x, cudaStream_t s) {
  if (!plan) return interp_only();
  NufftBatch b;
  b.C = 1;
  b.data_stride = plan->M;
  return nufft_adjoint(plan.get(), b, y, x, s);
}
uint64_t GnufftOp::resident_bytes() const {
  if (!plan) return interp ? interp->M * 16 + interp->lut.bytes() : 0;
  return plan->M * (3 * 4 + 8 + 64 + 4 + 4) + plan->work->grids.bytes() + plan->work->agrids.bytes() +
         plan->work->fin.bytes();
}

// ---- Gdft ------------------------------------------------------------------
pg_status GdftOp::forward(const float2* x, float2* y, cudaStream_t s) {
  return gdft_forward(plan.get(), 1, nullptr, x, y, plan->nk, s);
}
pg_status GdftOp::adjoint(const float2* y, float2* x, cudaStream_t s) {
  return gdft_adjoint(plan.get(), 1, nullptr, y, plan->nk, x, s);
}

// ---- TimeSegmentation --------------------------------------------------------
pg_status TimeSegOp::forward(const float2* x, float2* y, cudaStream_t s) {
  if (tab.L == 1) return inner->forward(x, y, s);  // AA = Wo = 1
  if (inner->kind == PG_OP_GNUFFT && bin) {
    auto* g = static_cast<GnufftOp*>(inner);
    NufftBatch b;
    b.C = 1;
    b.Wo = Wo.p;
    b.bin = bin.get();
    b.data_stride = n_data;
    return nufft_forward(g->plan.get(), b, x, y, s);
  }
  // generic: y = sum_l AA_l (.) G(Wo_l (.) x)   (TimeSegmentation.cpp:266-295)
  PG_TRY(grow(tmp_img, n_image, s));
  PG_TRY(grow(tmp_data, n_data, s));
  for (int l = 0; l < tab.L; ++l) {
    PG_LAUNCH(k_cmul, ceil_div(n_image, 256), 256, 0, s, n_image, Wo.p + (uint64_t)l * n_image, x, 0, tmp_img.p);
    PG_TRY(inner->forward(tmp_img.p, tmp_data.p, s));
    PG_LAUNCH(k_cmul_acc, ceil_div(n_data, 256), 256, 0, s, n_data, tmp_data.p, AAfull.p + (uint64_t)l * n_data, 0,
              l > 0 ? 1 : 0, y);
  }
  return PG_OK;
}
pg_status TimeSegOp::adjoint(const float2* y, float2* x, cudaStream_t s) {
  if (tab.L == 1) return inner->adjoint(y, x, s);
  if (inner->kind == PG_OP_GNUFFT && bin) {
    auto* g = static_cast<GnufftOp*>(inner);
    NufftBatch b;
    b.C = 1;
    b.WoH = WoH.p;
    b.bin = bin.get();
    b.data_stride = n_data;
    return nufft_adjoint(g->plan.get(), b, y, x, s);
  }
  // generic: x = sum_l WoH_l (.) G^H(conj(AA_l) (.) y)   (TimeSegmentation.cpp:304-323)
  PG_TRY(grow(tmp_img, n_image, s));
  PG_TRY(grow(tmp_data, n_data, s));
  for (int l = 0; l < tab.L; ++l) {
    PG_LAUNCH(k_cmul, ceil_div(n_data, 256), 256, 0, s, n_data, AAfull.p + (uint64_t)l * n_data, y, 1, tmp_data.p);
    PG_TRY(inner->adjoint(tmp_data.p, tmp_img.p, s));
    PG_LAUNCH(k_cmul_acc, ceil_div(n_image, 256), 256, 0, s, n_image, tmp_img.p, WoH.p + (uint64_t)l * n_image, 0,
              l > 0 ? 1 : 0, x);
  }
  return PG_OK;
}

// ---- SENSE -------------------------------------------------------------------
static bool nufft_under(pg_op_s* inner, NufftPlan** plan, const TimeSegOp** ts) {
  *ts = nullptr;
  if (inner->kind == PG_OP_GNUFFT) {
    *plan = static_cast<GnufftOp*>(inner)->plan.get();
    return *plan != nullptr;
  }
  if (inner->kind == PG_OP_TIMESEG) {
    auto* t = static_cast<TimeSegOp*>(inner);
    if (t->inner->kind == PG_OP_GNUFFT) {
      if (t->tab.L > 1 && !t->bin) return false;  // segments applied one at a time
      *plan = static_cast<GnufftOp*>(t->inner)->plan.get();
      *ts = t->tab.L > 1 ? t : nullptr;
      return *plan != nullptr;
    }
  }
  return false;
}

pg_status SenseOp::forward(const float2* x, float2* y, cudaStream_t s) {
  NufftPlan* plan = nullptr;
  const TimeSegOp* ts = nullptr;
  if (nufft_under(inner, &plan, &ts)) {
    NufftBatch b;
    b.C = (int)nc;
    b.S = S.p;
    b.data_stride = n_data / nc;  // per-coil data length (SENSE.cpp:86)
    if (ts) { b.Wo = ts->Wo.p; b.bin = ts->bin.get(); }
    return nufft_forward(plan, b, x, y, s);
  }
  if (inner->kind == PG_OP_GDFT)
    return gdft_forward(static_cast<GdftOp*>(inner)->plan.get(), (int)nc, S.p, x, y, n_data / nc, s);
  // generic (SENSE.cpp:59-70)
  PG_TRY(grow(tmp_img, n_image, s));
  for (uint64_t c = 0; c < nc; ++c) {
    PG_LAUNCH(k_cmul, ceil_div(n_image, 256), 256, 0, s, n_image, S.p + c * n_image, x, 0, tmp_img.p);
    PG_TRY(inner->forward(tmp_img.p, y + c * (n_data / nc), s));
  }
  return PG_OK;
}

pg_status SenseOp::adjoint(const float2* y, float2* x, cudaStream_t s) {
  NufftPlan* plan = nullptr;
  const TimeSegOp* ts = nullptr;
  if (nufft_under(inner, &plan, &ts)) {
    NufftBatch b;
    b.C = (int)nc;
    b.S = S.p;
    b.data_stride = n_data / nc;  // per-coil data length (SENSE.cpp:86)
    if (ts) { b.WoH = ts->WoH.p; b.bin = ts->bin.get(); }
    return nufft_adjoint(plan, b, y, x, s);
  }
  if (inner->kind == PG_OP_GDFT)
    return gdft_adjoint(static_cast<GdftOp*>(inner)->plan.get(), (int)nc, S.p, y, n_data / nc, x, s);
  // generic (SENSE.cpp:84-96)
  PG_TRY(grow(tmp_img, n_image, s));
  for (uint64_t c = 0; c < nc; ++c) {
    PG_TRY(inner->adjoint(y + c * (n_data / nc), tmp_img.p, s));
    PG_LAUNCH(k_cmul_acc, ceil_div(n_image, 256), 256, 0, s, n_image, tmp_img.p, S.p + c * n_image, 1,
              c > 0 ? 1 : 0, x);
  }
  return PG_OK;
}

// ---- pcSenseTimeSeg ----------------------------------------------------------
pg_status PcSenseTsOp::forward(const float2* x, float2* y, cudaStream_t s) {
  for (uint64_t sh = 0; sh < Ns; ++sh) {
    NufftBatch b;
    b.C = (int)Nc;
    b.S = S.p;
    b.E = E.p + sh * Ni;
    b.data_stride = Ns * Nd;
    if (tabs[sh].L > 1) { b.Wo = Wo[sh].p; b.bin = bins[sh].get(); }
    PG_TRY(nufft_forward(plans[sh].get(), b, x, y + sh * Nd, s));
  }
  return PG_OK;
}
pg_status PcSenseTsOp::adjoint(const float2* y, float2* x, cudaStream_t s) {
  for (uint64_t sh = 0; sh < Ns; ++sh) {
    NufftBatch b;
    b.C = (int)Nc;
    b.S = S.p;
    b.E = E.p + sh * Ni;
    b.data_stride = Ns * Nd;
    b.accumulate = sh > 0;
    if (tabs[sh].L > 1) { b.WoH = WoH[sh].p; b.bin = bins[sh].get(); }
    PG_TRY(nufft_adjoint(plans[sh].get(), b, y + sh * Nd, x, s));
  }
  return PG_OK;
}
uint64_t PcSenseTsOp::resident_bytes() const {
  uint64_t b = S.bytes() + E.bytes();
  for (auto& p : plans) b += p->M * 100;
  if (!plans.empty())
    b += plans[0]->work->grids.bytes() + plans[0]->work->agrids.bytes() + plans[0]->work->fin.bytes() +
         plans[0]->work->fft_work.bytes();
  return b;
}

// ---- pcSENSE (over Gdft) --------------------------------------------------------
// fwd column (s + c*Ns) = G_s (x (.) S_c (.) E_s)   (pcSENSE.cpp:113-126)
pg_status PcSenseOp::forward(const float2* x, float2* y, cudaStream_t s) {
  PG_TRY(grow(tmp, Ni, s));
  for (uint64_t sh = 0; sh < Ns; ++sh) {
    PG_LAUNCH(k_cmul, ceil_div(Ni, 256), 256, 0, s, Ni, E.p + sh * Ni, x, 0, tmp.p);
    PG_TRY(gdft_forward(plans[sh].get(), (int)Nc, S.p, tmp.p, y + sh * Nd, Ns * Nd, s));
  }
  return PG_OK;
}
// adj = sum_{c,s} conj(S_c) (.) E_s (.) G_s^H d_{c,s}   (pcSENSE.cpp:131-150): the
// phase factor is E_s in both directions, as in the reference.
pg_status PcSenseOp::adjoint(const float2* y, float2* x, cudaStream_t s) {
  PG_TRY(grow(tmp, Ni, s));
  for (uint64_t sh = 0; sh < Ns; ++sh) {
    PG_TRY(gdft_adjoint(plans[sh].get(), (int)Nc, S.p, y + sh * Nd, Ns * Nd, tmp.p, s));
    PG_LAUNCH(k_cmul_acc, ceil_div(Ni, 256), 256, 0, s, Ni, tmp.p, E.p + sh * Ni, 0, sh > 0 ? 1 : 0, x);
  }
  return PG_OK;
}
uint64_t PcSenseOp::resident_bytes() const {
  uint64_t b = S.bytes() + E.bytes() + tmp.bytes();
  for (auto& p : plans) b += p->ks.bytes() + (p->vs.owned ? p->vs.bytes() : 0);
  if (!plans.empty()) b += plans[0]->work->xin.bytes() + plans[0]->work->part.bytes();
  return b;
}

// ---------------------------------------------------------------------------
// LRobj (lowRank/LRobj.cpp:27-68)
// ---------------------------------------------------------------------------
namespace {
// Thread per output element; a transposed output puts a fastest across the
// threads (coalesced stores, the input reads broadcast within a pixel).
__global__ void k_mix_columns(uint64_t N, int Kin, int Kout, const float2* __restrict__ in,
                              const float2* __restrict__ C, int transposed_out, float2* __restrict__ out) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N * (uint64_t)Kout) return;
  uint64_t n;
  int a;
  if (transposed_out) { a = (int)(t % Kout); n = t / Kout; }
  else { n = t % N; a = (int)(t / N); }
  float2 acc = make_float2(0.f, 0.f);
  for (int b = 0; b < Kin; ++b) acc = cadd(acc, cmul(in[n + N * b], C[a + (uint64_t)Kout * b]));
  out[t] = acc;
}
}  // namespace

pg_status mix_columns(uint64_t N, int Kin, int Kout, const float2* in, const float2* C, bool transposed_out,
                      float2* out, cudaStream_t s) {
  const uint64_t n = N * (uint64_t)Kout;
  if (n == 0) return PG_OK;
  PG_LAUNCH(k_mix_columns, ceil_div(n, 256), 256, 0, s, N, Kin, Kout, in, C, transposed_out ? 1 : 0, out);
  return PG_OK;
}

pg_status LowRankOp::forward(const float2* x, float2* y, cudaStream_t s) {
  PG_TRY(stack.alloc(N * Ni));
  PG_TRY(mix_columns(N, (int)K, (int)Ni, x, cf.p, false, stack.p, s));
  for (uint64_t i = 0; i < Ni; ++i) PG_TRY(ops[i]->forward(stack.p + N * i, y + Nd * i, s));
  return PG_OK;
}

pg_status LowRankOp::adjoint(const float2* y, float2* x, cudaStream_t s) {
  PG_TRY(stack.alloc(N * Ni));
  for (uint64_t i = 0; i < Ni; ++i) PG_TRY(ops[i]->adjoint(y + Nd * i, stack.p + N * i, s));
  return mix_columns(N, (int)Ni, (int)K, stack.p, ca.p, false, x, s);
}

uint64_t LowRankOp::resident_bytes() const { return cf.bytes() + ca.bytes() + N * Ni * sizeof(float2); }

// The fused gridding stages K segment grids per tile in shared memory: up to
// 8 in-plane (the forward's register budget), 3 in 3-D (8x8x8 tiles padded
// to 16x24x16 complex cells, 48 KB each).  Wider windows (the dense min-max
// interpolators) apply the segments one at a time, as the reference does.
bool segment_window_fits(const NufftPlan& p, int K) { return p.g.dim == 2 ? K <= 8 : K <= 3; }

static pg_status make_binning_for(NufftPlan* plan, const TsTables& tab, std::unique_ptr<Binning>* out,
                                  cudaStream_t s) {
  return nufft_build_binning(plan, tab.L, tab.K, tab.l0.data(), tab.aa_win.data(), out, s);
}

pg_status make_gnufft(std::unique_ptr<GnufftOp>* out, uint64_t data_length, float gridos, uint64_t nx, uint64_t ny,
                      uint64_t nz, const float* kx, const float* ky, const float* kz, cudaStream_t s) {
  if (!kx || !ky) return set_error(PG_INVALID_ARG, "Gnufft: null argument");
  if (nz > 1 && !kz) return set_error(PG_INVALID_ARG, "Gnufft: kz required for 3-D");
  auto op = std::make_unique<GnufftOp>();
  op->kind = PG_OP_GNUFFT;
  if (gridos != 2.0f)
    PG_TRY(interp_plan_create(&op->interp, data_length, gridos, (int)nx, (int)ny, (int)nz, kx, ky, kz, s));
  else
    PG_TRY(nufft_plan_create(&op->plan, data_length, gridos, (int)nx, (int)ny, (int)nz, kx, ky, kz, s));
  op->n_data = data_length;
  op->n_image = nx * ny * nz;
  *out = std::move(op);
  return PG_OK;
}

pg_status make_timeseg(std::unique_ptr<TimeSegOp>* out, pg_op_s* G, const float* field_map, const float* tvec,
                       uint64_t n1, uint64_t n2, uint64_t L, uint64_t interptype, uint64_t shots, cudaStream_t s) {
  if (!G || !field_map || !tvec) return set_error(PG_INVALID_ARG, "TimeSegmentation: null argument");
  if (G->n_data != n1 || G->n_image != n2)
    return set_error(PG_INVALID_ARG, "TimeSegmentation: sizes (%llu, %llu) do not match the inner operator (%llu, %llu)",
                     (unsigned long long)n1, (unsigned long long)n2, (unsigned long long)G->n_data,
                     (unsigned long long)G->n_image);
  auto op = std::make_unique<TimeSegOp>();
  op->kind = PG_OP_TIMESEG;
  op->inner = G;
  op->n_data = n1;
  op->n_image = n2;
  PG_TRY(build_ts_tables(field_map, tvec, n1, n2, L, interptype, shots, &op->tab));
  if (op->tab.L > 1) {
    PG_TRY(build_ts_phases(op->tab, field_map, n2, &op->Wo, &op->WoH, s));
    NufftPlan* np = G->kind == PG_OP_GNUFFT ? static_cast<GnufftOp*>(G)->plan.get() : nullptr;
    if (G->kind == PG_OP_GNUFFT && !np) return interp_only();
    if (np && segment_window_fits(*np, op->tab.K)) {
      PG_TRY(make_binning_for(np, op->tab, &op->bin, s));
    } else {
      PG_TRY(op->AAfull.upload(op->tab.AA.data(), op->tab.AA.size(), s));
    }
  }
  PG_CUDA(cudaStreamSynchronize(s));
  // host tables are only needed to build the device ones
  op->tab.AA.clear(); op->tab.AA.shrink_to_fit();
  *out = std::move(op);
  return PG_OK;
}

pg_status make_gnufft_shared(std::unique_ptr<GnufftOp>* out, const GnufftOp& src) {
  auto op = std::make_unique<GnufftOp>();
  op->kind = PG_OP_GNUFFT;
  if (!src.plan) return interp_only();
  PG_TRY(nufft_plan_share(*src.plan, &op->plan));
  op->n_data = src.n_data;
  op->n_image = src.n_image;
  *out = std::move(op);
  return PG_OK;
}

pg_status make_timeseg_shared(std::unique_ptr<TimeSegOp>* out, pg_op_s* G, const TimeSegOp& src,
                              const float* field_map, cudaStream_t s) {
  if (!G || !field_map) return set_error(PG_INVALID_ARG, "TimeSegmentation: null argument");
  if (G->n_data != src.n_data || G->n_image != src.n_image)
    return set_error(PG_INVALID_ARG, "TimeSegmentation: shared tables do not match the inner operator");
  for (uint64_t p = 0; p < src.n_image; ++p)
    if (!std::isfinite(field_map[p])) return set_error(PG_INVALID_ARG, "TimeSegmentation: non-finite field map");
  auto op = std::make_unique<TimeSegOp>();
  op->kind = PG_OP_TIMESEG;
  op->inner = G;
  op->n_data = src.n_data;
  op->n_image = src.n_image;
  op->tab.L = src.tab.L;
  op->tab.tau = src.tab.tau;
  op->tab.tmin = src.tab.tmin;
  op->tab.K = src.tab.K;
  if (op->tab.L > 1) {
    PG_TRY(build_ts_phases(op->tab, field_map, op->n_image, &op->Wo, &op->WoH, s));
    if (src.bin) op->bin = binning_share(*src.bin);
    if (src.AAfull.p) op->AAfull.borrow(src.AAfull);
  }
  *out = std::move(op);
  return PG_OK;
}

// ---- the slices of a request as one operator ---------------------------------
pg_status make_slice_batch(std::unique_ptr<SliceBatchOp>* out, GnufftOp* G, const TimeSegOp* ts, uint64_t ns,
                           uint64_t nc, const float* const* field_maps, const float* const* sense_maps,
                           cudaStream_t s) {
  if (!G || !G->plan || !sense_maps || (ts && !field_maps) || ns == 0 || nc == 0)
    return set_error(PG_INVALID_ARG, "slice batch: null argument");
  const uint64_t N = G->n_image, M = G->n_data;
  auto op = std::make_unique<SliceBatchOp>();
  op->kind = PG_OP_SENSE;
  op->G = G;
  op->ts = (ts && ts->tab.L > 1) ? ts : nullptr;
  op->ns = ns;
  op->nc = nc;
  op->N = N;
  op->M = M;
  op->L = op->ts ? op->ts->tab.L : 1;
  op->n_image = ns * N;
  op->n_data = ns * nc * M;
  op->n_seg = ns;
  for (uint64_t sl = 0; sl < ns; ++sl)
    if (!sense_maps[sl] || (op->ts && !field_maps[sl])) return set_error(PG_INVALID_ARG, "slice batch: null map");
  if (op->ts) {
    if (ts->n_image != N || ts->n_data != M || !ts->bin)
      return set_error(PG_INVALID_ARG, "slice batch: segmentation does not match the Gnufft");
    for (uint64_t sl = 0; sl < ns; ++sl)
      for (uint64_t p = 0; p < N; ++p)
        if (!std::isfinite(field_maps[sl][p])) return set_error(PG_INVALID_ARG, "slice batch: non-finite field map");
    DevBuf<float> fm;
    PG_TRY(fm.alloc(ns * N));
    for (uint64_t sl = 0; sl < ns; ++sl)
      PG_CUDA(cudaMemcpyAsync(fm.p + sl * N, field_maps[sl], N * sizeof(float), cudaMemcpyHostToDevice, s));
    const uint64_t LN = (uint64_t)op->L * N;
    PG_TRY(op->Wo.alloc(ns * LN));
    PG_TRY(op->WoH.alloc(ns * LN));
    for (uint64_t sl = 0; sl < ns; ++sl)
      PG_LAUNCH(k_ts_phases, ceil_div(LN, 256), 256, 0, s, N, op->L, ts->tab.tau, ts->tab.tmin, fm.p + sl * N,
                op->Wo.p + sl * LN, op->WoH.p + sl * LN);
    PG_CUDA(cudaStreamSynchronize(s));  // fm is released on return
  }
  PG_TRY(op->S.alloc(ns * nc * N));
  for (uint64_t sl = 0; sl < ns; ++sl)
    PG_CUDA(cudaMemcpyAsync(op->S.p + sl * nc * N, sense_maps[sl], nc * N * sizeof(float2), cudaMemcpyHostToDevice,
                            s));
  PG_CUDA(cudaStreamSynchronize(s));  // the host maps may be released on return
  *out = std::move(op);
  return PG_OK;
}

pg_status SliceBatchOp::forward(const float2* x, float2* y, cudaStream_t s) {
  NufftBatch b;
  b.C = (int)(ns * nc);
  b.S = S.p;
  b.data_stride = M;
  b.cgroup = (int)nc;
  b.image_stride = N;
  b.phase_stride = (uint64_t)L * N;
  if (ts) { b.Wo = Wo.p; b.bin = ts->bin.get(); }
  return nufft_forward(G->plan.get(), b, x, y, s);
}

pg_status SliceBatchOp::adjoint(const float2* y, float2* x, cudaStream_t s) {
  NufftBatch b;
  b.C = (int)(ns * nc);
  b.S = S.p;
  b.data_stride = M;
  b.cgroup = (int)nc;
  b.image_stride = N;
  b.phase_stride = (uint64_t)L * N;
  if (ts) { b.WoH = WoH.p; b.bin = ts->bin.get(); }
  return nufft_adjoint(G->plan.get(), b, y, x, s);
}

pg_status tune_for_coils(pg_op_s* G, int nc, bool search, cudaStream_t s) {
  if (G->kind == PG_OP_GNUFFT) {
    NufftPlan* plan = static_cast<GnufftOp*>(G)->plan.get();
    if (!plan) return PG_OK;
    return nufft_autotune(plan, 1, 1, nullptr, nullptr, nc, &plan->plain, search, s);
  }
  if (G->kind == PG_OP_TIMESEG) {
    auto* t = static_cast<TimeSegOp*>(G);
    // operators sharing another one's tables inherit its tuning
    if (t->inner->kind != PG_OP_GNUFFT || t->tab.L <= 1 || t->tab.l0.empty() || !t->bin) return PG_OK;
    NufftPlan* plan = static_cast<GnufftOp*>(t->inner)->plan.get();
    return nufft_autotune(plan, t->tab.L, t->tab.K, t->tab.l0.data(), t->tab.aa_win.data(), nc, &t->bin, search,
                          s);
  }
  return PG_OK;
}

pg_status make_sense(std::unique_ptr<SenseOp>* out, pg_op_s* G, const float* sense_map, uint64_t n1, uint64_t n2,
                     uint64_t nc, cudaStream_t s) {
  if (!G || !sense_map) return set_error(PG_INVALID_ARG, "SENSE: null argument");
  if (nc == 0) return set_error(PG_INVALID_ARG, "SENSE: nc = 0");
  if (G->n_data != n1 || G->n_image != n2) return set_error(PG_INVALID_ARG, "SENSE: sizes do not match the inner operator");
  auto op = std::make_unique<SenseOp>();
  op->kind = PG_OP_SENSE;
  op->inner = G;
  op->nc = nc;
  op->n_data = n1 * nc;
  op->n_image = n2;
  PG_TRY(op->S.upload(reinterpret_cast<const float2*>(sense_map), n2 * nc, s));
  PG_TRY(tune_for_coils(G, (int)nc, true, s));
  PG_CUDA(cudaStreamSynchronize(s));
  *out = std::move(op);
  return PG_OK;
}

}  // namespace pg

using namespace pg;

// ---- C ABI -------------------------------------------------------------------
extern "C" {

pg_status pg_gnufft_create(pg_op* out, uint64_t data_length, float gridos, uint64_t nx, uint64_t ny, uint64_t nz,
                           const float* kx, const float* ky, const float* kz) {
  if (!out) return set_error(PG_INVALID_ARG, "Gnufft: null argument");
  PG_TRY(ensure_init());
  std::unique_ptr<GnufftOp> op;
  PG_TRY(make_gnufft(&op, data_length, gridos, nx, ny, nz, kx, ky, kz, default_stream()));
  *out = op.release();
  return PG_OK;
}

pg_status pg_gdft_create(pg_op* out, uint64_t nk, uint64_t ni, const float* kx, const float* ky, const float* kz,
                         const float* ix, const float* iy, const float* iz, const float* field_map, const float* t) {
  if (!out || !kx || !ky || !kz || !ix || !iy || !iz || !field_map || !t)
    return set_error(PG_INVALID_ARG, "Gdft: null argument");
  PG_TRY(ensure_init());
  auto op = std::make_unique<GdftOp>();
  op->kind = PG_OP_GDFT;
  PG_TRY(gdft_plan_create(&op->plan, nk, ni, kx, ky, kz, ix, iy, iz, field_map, t, default_stream()));
  op->n_data = nk;
  op->n_image = ni;
  *out = op.release();
  return PG_OK;
}

pg_status pg_gdftr2_create(pg_op* out, uint64_t nk, uint64_t ni, const float* kx, const float* ky, const float* kz,
                           const float* ix, const float* iy, const float* iz, const float* field_map, const float* t,
                           uint64_t nx, uint64_t ny, uint64_t nz) {
  if (!out || !kx || !ky || !kz || !ix || !iy || !iz || !field_map || !t)
    return set_error(PG_INVALID_ARG, "GdftR2: null argument");
  PG_TRY(ensure_init());
  auto op = std::make_unique<GdftOp>();
  op->kind = PG_OP_GDFT;
  cudaStream_t s = default_stream();
  PG_TRY(gdft_plan_create(&op->plan, nk, ni, kx, ky, kz, ix, iy, iz, field_map, t, s));
  PG_TRY(gdft_plan_add_gradients(op->plan.get(), kx, ky, kz, t, field_map, (int)nx, (int)ny, (int)nz, s));
  op->n_data = nk;
  op->n_image = ni;
  *out = op.release();
  return PG_OK;
}

pg_status pg_timeseg_create(pg_op* out, pg_op G, const float* field_map, const float* tvec, uint64_t n1, uint64_t n2,
                            uint64_t L, uint64_t interptype, uint64_t shots) {
  if (!out) return set_error(PG_INVALID_ARG, "TimeSegmentation: null argument");
  PG_TRY(ensure_init());
  std::unique_ptr<TimeSegOp> op;
  PG_TRY(make_timeseg(&op, G, field_map, tvec, n1, n2, L, interptype, shots, default_stream()));
  *out = op.release();
  return PG_OK;
}

pg_status pg_sense_create(pg_op* out, pg_op G, const float* sense_map, uint64_t n1, uint64_t n2, uint64_t nc) {
  if (!out) return set_error(PG_INVALID_ARG, "SENSE: null argument");
  PG_TRY(ensure_init());
  std::unique_ptr<SenseOp> op;
  PG_TRY(make_sense(&op, G, sense_map, n1, n2, nc, default_stream()));
  *out = op.release();
  return PG_OK;
}

pg_status pg_pcsense_timeseg_create(pg_op* out, const float* kx, const float* ky, const float* kz, uint64_t nk,
                                    uint64_t nx, uint64_t ny, uint64_t nz, uint64_t nc, const float* t, uint64_t L,
                                    uint64_t interptype, const float* sense_map, const float* field_map,
                                    const float* shot_phase_map, uint64_t n_shot_phase) {
  if (!out || !kx || !ky || !kz || !t || !sense_map || !field_map || !shot_phase_map)
    return set_error(PG_INVALID_ARG, "pcSenseTimeSeg: null argument");
  PG_TRY(ensure_init());
  const uint64_t Ni = nx * ny * nz;
  if (Ni == 0 || n_shot_phase % Ni) return set_error(PG_INVALID_ARG, "pcSenseTimeSeg: phase map size");
  const uint64_t Ns = n_shot_phase / Ni;  // pcSenseTimeSeg.cpp:47
  if (Ns == 0 || nk % Ns) return set_error(PG_INVALID_ARG, "pcSenseTimeSeg: samples not divisible by shots");
  const uint64_t Nd = nk / Ns;            // :48
  auto op = std::make_unique<PcSenseTsOp>();
  op->kind = PG_OP_PCSENSE_TS;
  op->Ni = Ni; op->Nc = nc; op->Ns = Ns; op->Nd = Nd;
  op->n_data = Nd * Ns * nc;
  op->n_image = Ni;
  cudaStream_t s = default_stream();
  op->Wo.resize(Ns);
  op->WoH.resize(Ns);
  op->tabs.resize(Ns);
  op->bins.resize(Ns);
  for (uint64_t sh = 0; sh < Ns; ++sh) {
    std::unique_ptr<NufftPlan> plan;
    PG_TRY(nufft_plan_create(&plan, Nd, 2.0f, (int)nx, (int)ny, (int)nz, kx + sh * Nd, ky + sh * Nd, kz + sh * Nd, s));
    PG_TRY(build_ts_tables(field_map, t + sh * Nd, Nd, Ni, L, interptype, 1, &op->tabs[sh]));
    if (op->tabs[sh].L > 1) {
      if (!segment_window_fits(*plan, op->tabs[sh].K))
        return set_error(PG_INVALID_ARG, "pcSenseTimeSeg: interpolator spans %d segments per sample; the fused "
                                         "gridding takes at most %d here", op->tabs[sh].K, plan->g.dim == 2 ? 8 : 3);
      PG_TRY(build_ts_phases(op->tabs[sh], field_map, Ni, &op->Wo[sh], &op->WoH[sh], s));
      PG_TRY(nufft_autotune(plan.get(), op->tabs[sh].L, op->tabs[sh].K, op->tabs[sh].l0.data(),
                            op->tabs[sh].aa_win.data(), (int)nc, &op->bins[sh], true, s));
      op->tabs[sh].AA.clear();
      op->tabs[sh].AA.shrink_to_fit();
    }
    // the shots run one after another on one stream: one grid workspace serves all
    if (sh > 0) plan->work = op->plans[0]->work;
    op->plans.push_back(std::move(plan));
  }
  PG_TRY(op->S.upload(reinterpret_cast<const float2*>(sense_map), Ni * nc, s));
  // E_s = exp(-i P_s) (pcSenseTimeSeg.cpp:107)
  std::vector<float2> E(Ni * Ns);
  for (uint64_t i = 0; i < Ni * Ns; ++i) {
    const float ph = shot_phase_map[i];
    if (!std::isfinite(ph)) return set_error(PG_INVALID_ARG, "pcSenseTimeSeg: non-finite phase map");
    E[i] = make_float2(std::cos(ph), -std::sin(ph));
  }
  PG_TRY(op->E.upload(E.data(), E.size(), s));
  PG_CUDA(cudaStreamSynchronize(s));
  *out = op.release();
  return PG_OK;
}

pg_status pg_pcsense_create(pg_op* out, const float* kx, const float* ky, const float* kz, uint64_t nk, uint64_t nx,
                            uint64_t ny, uint64_t nz, uint64_t nc, const float* t, const float* sense_map,
                            const float* field_map, const float* shot_phase_map, uint64_t n_shot_phase) {
  if (!out || !kx || !ky || !kz || !t || !sense_map || !field_map || !shot_phase_map)
    return set_error(PG_INVALID_ARG, "pcSENSE: null argument");
  PG_TRY(ensure_init());
  const uint64_t Ni = nx * ny * nz;
  if (Ni == 0 || n_shot_phase % Ni) return set_error(PG_INVALID_ARG, "pcSENSE: phase map size");
  const uint64_t Ns = n_shot_phase / Ni;  // pcSENSE.cpp:44
  if (Ns == 0 || nk % Ns) return set_error(PG_INVALID_ARG, "pcSENSE: samples not divisible by shots");
  if (nc == 0) return set_error(PG_INVALID_ARG, "pcSENSE: no coils");
  const uint64_t Nd = nk / Ns;            // :45
  auto op = std::make_unique<PcSenseOp>();
  op->kind = PG_OP_PCSENSE;
  op->Ni = Ni; op->Nc = nc; op->Ns = Ns; op->Nd = Nd;
  op->n_data = Nd * Ns * nc;
  op->n_image = Ni;
  cudaStream_t s = default_stream();
  // voxel coordinates (pcSENSE.cpp:65-82): ix = (x - Nx/2)/Nx evaluated with a
  // double Nx/2, y fastest
  std::vector<float> ix(Ni), iy(Ni), iz(Ni);
  for (uint64_t z = 0; z < nz; ++z)
    for (uint64_t xx = 0; xx < nx; ++xx)
      for (uint64_t yy = 0; yy < ny; ++yy) {
        const uint64_t j = yy + ny * (xx + nx * z);
        ix[j] = (float)(((float)xx - (float)nx / 2.0) / ((float)nx));
        iy[j] = (float)(((float)yy - (float)ny / 2.0) / ((float)ny));
        iz[j] = (float)(((float)z - (float)nz / 2.0) / ((float)nz));
      }
  for (uint64_t sh = 0; sh < Ns; ++sh) {
    std::unique_ptr<GdftPlan> plan;
    if (sh == 0)
      PG_TRY(gdft_plan_create(&plan, Nd, Ni, kx, ky, kz, ix.data(), iy.data(), iz.data(), field_map, t, s));
    else
      PG_TRY(gdft_plan_same_voxels(&plan, *op->plans[0], Nd, kx + sh * Nd, ky + sh * Nd, kz + sh * Nd, t + sh * Nd,
                                   s));
    op->plans.push_back(std::move(plan));
  }
  PG_TRY(op->S.upload(reinterpret_cast<const float2*>(sense_map), Ni * nc, s));
  std::vector<float2> E(Ni * Ns);
  for (uint64_t i = 0; i < Ni * Ns; ++i) {
    const float ph = shot_phase_map[i];
    if (!std::isfinite(ph)) return set_error(PG_INVALID_ARG, "pcSENSE: non-finite phase map");
    E[i] = make_float2(std::cos(ph), std::sin(ph));
  }
  PG_TRY(op->E.upload(E.data(), E.size(), s));
  PG_CUDA(cudaStreamSynchronize(s));
  *out = op.release();
  return PG_OK;
}

pg_status pg_lowrank_create(pg_op* out, uint64_t n_image, uint64_t n_data, uint64_t rank, uint64_t n_img,
                            const float* v, const pg_op* ops) {
  if (!out || !v || !ops) return set_error(PG_INVALID_ARG, "LRobj: null argument");
  if (rank == 0 || n_img == 0 || n_image == 0 || n_data == 0)
    return set_error(PG_INVALID_ARG, "LRobj: empty model (rank %llu, %llu images)", (unsigned long long)rank,
                     (unsigned long long)n_img);
  if (rank > 1024 || n_img > 65536) return set_error(PG_INVALID_ARG, "LRobj: rank or image count too large");
  for (uint64_t i = 0; i < n_img; ++i) {
    if (!ops[i]) return set_error(PG_INVALID_ARG, "LRobj: operator %llu is null", (unsigned long long)i);
    if (ops[i]->n_image != n_image || ops[i]->n_data != n_data)
      return set_error(PG_INVALID_ARG, "LRobj: operator %llu is %llux%llu, the model needs %llux%llu",
                       (unsigned long long)i, (unsigned long long)ops[i]->n_data,
                       (unsigned long long)ops[i]->n_image, (unsigned long long)n_data,
                       (unsigned long long)n_image);
  }
  PG_TRY(ensure_init());
  auto op = std::make_unique<LowRankOp>();
  op->kind = PG_OP_LOWRANK;
  op->N = n_image; op->Nd = n_data; op->K = rank; op->Ni = n_img;
  op->n_image = n_image * rank;   // LRobj.cpp:42 reshapes d to N x Nrank
  op->n_data = n_data * n_img;    // :43 (Ndata x Nimg)
  op->ops.assign(ops, ops + n_img);
  const float2* vb = reinterpret_cast<const float2*>(v);
  std::vector<float2> cf(n_img * rank), ca(rank * n_img);
  for (uint64_t k = 0; k < rank; ++k)
    for (uint64_t i = 0; i < n_img; ++i) {
      const float2 e = vb[k + rank * i];
      cf[i + n_img * k] = e;
      ca[k + rank * i] = make_float2(e.x, -e.y);
    }
  cudaStream_t s = default_stream();
  PG_TRY(op->cf.upload(cf.data(), cf.size(), s));
  PG_TRY(op->ca.upload(ca.data(), ca.size(), s));
  PG_TRY(op->stack.alloc(n_image * n_img));
  PG_CUDA(cudaStreamSynchronize(s));
  *out = op.release();
  return PG_OK;
}

pg_status pg_op_destroy(pg_op op) {
  if (!op) return PG_OK;
  // the operator may have been used on any stream; its buffers must be idle
  cudaDeviceSynchronize();
  delete op;
  return PG_OK;
}

pg_status pg_op_shape(pg_op op, uint64_t* n_data, uint64_t* n_image) {
  if (!op) return set_error(PG_INVALID_ARG, "null operator");
  if (n_data) *n_data = op->n_data;
  if (n_image) *n_image = op->n_image;
  return PG_OK;
}

pg_status pg_op_forward_device(pg_op op, const void* x, void* y, void* stream) {
  if (!op || !x || !y) return set_error(PG_INVALID_ARG, "forward: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  return op->forward((const float2*)x, (float2*)y, s);
}

pg_status pg_op_adjoint_device(pg_op op, const void* y, void* x, void* stream) {
  if (!op || !x || !y) return set_error(PG_INVALID_ARG, "adjoint: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = stream ? (cudaStream_t)stream : default_stream();
  return op->adjoint((const float2*)y, (float2*)x, s);
}

pg_status pg_op_forward(pg_op op, const float* x, float* y) {
  if (!op || !x || !y) return set_error(PG_INVALID_ARG, "forward: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  PG_TRY(op->hx.alloc(op->n_image));
  PG_TRY(op->hy.alloc(op->n_data));
  PG_CUDA(cudaMemcpyAsync(op->hx.p, x, op->n_image * sizeof(float2), cudaMemcpyHostToDevice, s));
  PG_TRY(op->forward(op->hx.p, op->hy.p, s));
  PG_CUDA(cudaMemcpyAsync(y, op->hy.p, op->n_data * sizeof(float2), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

pg_status pg_op_adjoint(pg_op op, const float* y, float* x) {
  if (!op || !x || !y) return set_error(PG_INVALID_ARG, "adjoint: null argument");
  PG_TRY(ensure_init());
  cudaStream_t s = default_stream();
  PG_TRY(op->hx.alloc(op->n_image));
  PG_TRY(op->hy.alloc(op->n_data));
  PG_CUDA(cudaMemcpyAsync(op->hy.p, y, op->n_data * sizeof(float2), cudaMemcpyHostToDevice, s));
  PG_TRY(op->adjoint(op->hy.p, op->hx.p, s));
  PG_CUDA(cudaMemcpyAsync(x, op->hx.p, op->n_image * sizeof(float2), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  return PG_OK;
}

uint64_t pg_util_kb_lut(float gridos, float* lut_out, uint64_t cap, float* beta_out) {
  std::vector<float> lut;
  float beta = 0.f;
  kb_table(gridos, &lut, &beta);
  if (beta_out) *beta_out = beta;
  if (lut_out) std::memcpy(lut_out, lut.data(), std::min<uint64_t>(cap, lut.size()) * sizeof(float));
  return lut.size();
}

pg_status pg_util_gnufft_binning(pg_op G, uint32_t* keys_out, uint32_t* perm_out, uint64_t* n_bins_out) {
  if (!G) return set_error(PG_INVALID_ARG, "null operator");
  const Binning* b = nullptr;
  if (G->kind == PG_OP_GNUFFT) {
    if (!static_cast<GnufftOp*>(G)->plan) return interp_only();
    PG_TRY(nufft_plain_binning(static_cast<GnufftOp*>(G)->plan.get(), default_stream()));
    b = static_cast<GnufftOp*>(G)->plan->plain.get();
  }
  else if (G->kind == PG_OP_TIMESEG && static_cast<TimeSegOp*>(G)->bin) b = static_cast<TimeSegOp*>(G)->bin.get();
  if (!b) return set_error(PG_INVALID_ARG, "operator has no sample binning");
  cudaStream_t s = default_stream();
  if (keys_out)
    PG_CUDA(cudaMemcpyAsync(keys_out, b->keys.p, b->M * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  if (perm_out)
    PG_CUDA(cudaMemcpyAsync(perm_out, b->perm.p, b->M * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  PG_CUDA(cudaStreamSynchronize(s));
  if (n_bins_out) *n_bins_out = b->nkeys;
  return PG_OK;
}

}  // extern "C"
