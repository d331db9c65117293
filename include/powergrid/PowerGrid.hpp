// PowerGrid operator API on the B200 library (header-only C++ over the C ABI
// in powergrid_b200.h).  Drop-in for the reference's
//   Gnufft<T1>            Gnufft.h:51-53
//   Gdft<T1>              Gdft.h:47-49
//   TimeSegmentation<T1, Tobj>   TimeSegmentation.h:70-71
//   SENSE<T1, Tobj>       SENSE.h:64
//   pcSenseTimeSeg<T1>    pcSenseTimeSeg.h:80-82
//   pcSENSE<T1>           pcSENSE.h:76-78
//   LRobj<T1, Gobj>       lowRank/LRobj.h:55
//   QuadPenalty<T1>, TVPenalty<T1>   QuadPenalty.h:43, TVPenalty.h:42
//   R_lowRank<T1, Robj>   lowRank/R_lowRank.h:52
//   solve_pwls_pcg        solve_pwls_pcg.hpp:48-51
//   reconSolve            reconSolve.h:63-66
//   acqTracking, getCompleteISMRMRDAcqData   acqTracking.h:14, processIsmrmrd.hpp:361-471
//   writeNiftiRealImage, writeNiftiMagPhsImage   processNIFTI.hpp:37-117
//   Server                (no counterpart: the request server over pg_server_*)
// with T1 = float.  Column types: any type with memptr() (or data()),
// n_elem (or size()) and a size constructor — arma::Col<std::complex<float>>
// and arma::Col<float> work unchanged; pg::Col<T> is provided for callers
// without Armadillo.  operator* / operator/ return new columns.
//
// Lifetimes follow the reference: composites keep a non-owning pointer to the
// operator they wrap (TimeSegmentation.cpp:53, SENSE.cpp:39).  Errors throw
// pg::Error (the reference printed and called exit(1)).
#pragma once

#include <complex>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../powergrid_b200.h"

namespace pg {

typedef unsigned long long uword;

struct Error : std::runtime_error {
  pg_status status;
  Error(pg_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(pg_status s) {
  if (s != PG_OK) throw Error(s, std::string(pg_status_string(s)) + ": " + pg_last_error());
}

// Minimal column vector for callers without Armadillo.
template <typename T>
class Col {
 public:
  Col() = default;
  explicit Col(uword n) : v_(n) {}
  Col(uword n, const T& fill) : v_(n, fill) {}
  T* memptr() { return v_.data(); }
  const T* memptr() const { return v_.data(); }
  uword n_elem_() const { return v_.size(); }
  T& operator()(uword i) { return v_[i]; }
  const T& operator()(uword i) const { return v_[i]; }
  T& operator[](uword i) { return v_[i]; }
  const T& operator[](uword i) const { return v_[i]; }
  uword size() const { return v_.size(); }

 private:
  std::vector<T> v_;
};

namespace detail {
template <typename C>
auto ptr(const C& c) -> decltype(c.memptr()) { return c.memptr(); }
template <typename C>
auto mptr(C& c) -> decltype(c.memptr()) { return c.memptr(); }
template <typename C>
uword len(const C& c) { return (uword)c.size(); }
}  // namespace detail

// Common operator base: owns the handle, provides operator* and operator/.
class Operator {
 public:
  Operator(const Operator&) = delete;
  Operator& operator=(const Operator&) = delete;
  virtual ~Operator() { if (h_) pg_op_destroy(h_); }
  pg_op handle() const { return h_; }
  uword n_data() const { return nd_; }
  uword n_image() const { return ni_; }

  template <typename CxCol>
  CxCol operator*(const CxCol& d) const {
    if (detail::len(d) != ni_) throw Error(PG_INVALID_ARG, "operator*: image length mismatch");
    CxCol out(nd_);
    check(pg_op_forward(h_, reinterpret_cast<const float*>(detail::ptr(d)),
                        reinterpret_cast<float*>(detail::mptr(out))));
    return out;
  }
  template <typename CxCol>
  CxCol operator/(const CxCol& d) const {
    if (detail::len(d) != nd_) throw Error(PG_INVALID_ARG, "operator/: data length mismatch");
    CxCol out(ni_);
    check(pg_op_adjoint(h_, reinterpret_cast<const float*>(detail::ptr(d)),
                        reinterpret_cast<float*>(detail::mptr(out))));
    return out;
  }

 protected:
  Operator() = default;
  void adopt(pg_op h) {
    h_ = h;
    uint64_t a = 0, b = 0;
    check(pg_op_shape(h_, &a, &b));
    nd_ = a;
    ni_ = b;
  }
  pg_op h_ = nullptr;
  uword nd_ = 0, ni_ = 0;
};

template <typename T1>
class Gnufft : public Operator {
  static_assert(std::is_same<T1, float>::value, "the B200 path computes in complex64");

 public:
  template <typename RCol>
  Gnufft(uword dataLength, T1 gridos, uword nx, uword ny, uword nz, const RCol& k1, const RCol& k2, const RCol& k3,
         const RCol& /*i1*/, const RCol& /*i2*/, const RCol& /*i3*/) {
    pg_op h = nullptr;
    check(pg_gnufft_create(&h, dataLength, gridos, nx, ny, nz, detail::ptr(k1), detail::ptr(k2), detail::ptr(k3)));
    adopt(h);
  }
  // Gnufft::forwardSpatialInterp / adjointSpatialInterp (Gnufft.cpp:213-337):
  // the oversampled grid in the reference's layout, no FFT.
  uword grid_length() const {
    uint64_t n = 0;
    check(pg_gnufft_grid_length(h_, &n));
    return n;
  }
  template <typename CxCol>
  CxCol forwardSpatialInterp(const CxCol& grid) const {
    if (detail::len(grid) != grid_length()) throw Error(PG_INVALID_ARG, "forwardSpatialInterp: grid length");
    CxCol out(nd_);
    check(pg_gnufft_forward_spatial_interp(h_, reinterpret_cast<const float*>(detail::ptr(grid)),
                                           reinterpret_cast<float*>(detail::mptr(out))));
    return out;
  }
  template <typename CxCol>
  CxCol adjointSpatialInterp(const CxCol& d) const {
    if (detail::len(d) != nd_) throw Error(PG_INVALID_ARG, "adjointSpatialInterp: data length");
    CxCol out(grid_length());
    check(pg_gnufft_adjoint_spatial_interp(h_, reinterpret_cast<const float*>(detail::ptr(d)),
                                           reinterpret_cast<float*>(detail::mptr(out))));
    return out;
  }
};

template <typename T1>
class Gdft : public Operator {
 public:
  template <typename RCol>
  Gdft(uword nk, uword ni, const RCol& k1, const RCol& k2, const RCol& k3, const RCol& i1, const RCol& i2,
       const RCol& i3, const RCol& FM, const RCol& t) {
    pg_op h = nullptr;
    check(pg_gdft_create(&h, nk, ni, detail::ptr(k1), detail::ptr(k2), detail::ptr(k3), detail::ptr(i1),
                         detail::ptr(i2), detail::ptr(i3), detail::ptr(FM), detail::ptr(t)));
    adopt(h);
  }
};

template <typename T1>
class GdftR2 : public Operator {
 public:
  template <typename RCol>
  GdftR2(uword nk, uword ni, const RCol& k1, const RCol& k2, const RCol& k3, const RCol& i1, const RCol& i2,
         const RCol& i3, const RCol& FM, const RCol& t, int num_x, int num_y, int num_z) {
    pg_op h = nullptr;
    check(pg_gdftr2_create(&h, nk, ni, detail::ptr(k1), detail::ptr(k2), detail::ptr(k3), detail::ptr(i1),
                           detail::ptr(i2), detail::ptr(i3), detail::ptr(FM), detail::ptr(t), num_x, num_y, num_z));
    adopt(h);
  }
};

template <typename T1, typename Tobj>
class TimeSegmentation : public Operator {
 public:
  template <typename RCol>
  TimeSegmentation(Tobj& G, const RCol& fieldMap, const RCol& timeVec, uword n1, uword n2, uword L,
                   uword interptype = 1, uword shots = 1) {
    pg_op h = nullptr;
    check(pg_timeseg_create(&h, G.handle(), detail::ptr(fieldMap), detail::ptr(timeVec), n1, n2, L, interptype,
                            shots));
    adopt(h);
  }
};

template <typename T1, typename Tobj>
class SENSE : public Operator {
 public:
  template <typename CxCol>
  SENSE(Tobj& G, const CxCol& senseMap, uword n1, uword n2, uword nc) {
    pg_op h = nullptr;
    check(pg_sense_create(&h, G.handle(), reinterpret_cast<const float*>(detail::ptr(senseMap)), n1, n2, nc));
    adopt(h);
  }
};

template <typename T1>
class pcSenseTimeSeg : public Operator {
 public:
  template <typename RCol, typename CxCol>
  pcSenseTimeSeg(const RCol& kx, const RCol& ky, const RCol& kz, uword nx, uword ny, uword nz, uword nc,
                 const RCol& t, uword L, uword intType, const CxCol& SENSEmap, const RCol& FieldMap,
                 const RCol& ShotPhaseMap) {
    pg_op h = nullptr;
    check(pg_pcsense_timeseg_create(&h, detail::ptr(kx), detail::ptr(ky), detail::ptr(kz), detail::len(kx), nx, ny,
                                    nz, nc, detail::ptr(t), L, intType,
                                    reinterpret_cast<const float*>(detail::ptr(SENSEmap)), detail::ptr(FieldMap),
                                    detail::ptr(ShotPhaseMap), detail::len(ShotPhaseMap)));
    adopt(h);
  }
};

template <typename T1>
class pcSENSE : public Operator {
 public:
  template <typename RCol, typename CxCol>
  pcSENSE(const RCol& kx, const RCol& ky, const RCol& kz, uword nx, uword ny, uword nz, uword nc, const RCol& t,
          const CxCol& SENSEmap, const RCol& FieldMap, const RCol& ShotPhaseMap) {
    pg_op h = nullptr;
    check(pg_pcsense_create(&h, detail::ptr(kx), detail::ptr(ky), detail::ptr(kz), detail::len(kx), nx, ny, nz, nc,
                            detail::ptr(t), reinterpret_cast<const float*>(detail::ptr(SENSEmap)),
                            detail::ptr(FieldMap), detail::ptr(ShotPhaseMap), detail::len(ShotPhaseMap)));
    adopt(h);
  }
};

// LRobj(NimgSize, N_data, n_rank, n_img, vBasis, All) (lowRank/LRobj.h:55):
// vBasis is n_rank x n_img (any column-major matrix with memptr()); All holds
// n_img operators, borrowed as the reference's raw pointers are.
template <typename T1, typename Gobj>
class LRobj : public Operator {
 public:
  template <typename CxMat>
  LRobj(uword NimgSize, uword N_data, uword n_rank, uword n_img, const CxMat& vBasis, Gobj** All) {
    std::vector<pg_op> ops(n_img);
    for (uword i = 0; i < n_img; ++i) ops[i] = All[i]->handle();
    pg_op h = nullptr;
    check(pg_lowrank_create(&h, NimgSize, N_data, n_rank, n_img,
                            reinterpret_cast<const float*>(detail::ptr(vBasis)), ops.data()));
    adopt(h);
  }
};

// calc3DDensityCompensation (reconSupport/directRecon.cpp:28-61).
template <typename T1, typename RCol>
RCol calc3DDensityCompensation(const RCol& kx, const RCol& ky, const RCol& kz, uword Ninplane, uword Nz) {
  RCol dcf(detail::len(kx));
  check(pg_density_compensation(detail::ptr(kx), detail::ptr(ky), detail::ptr(kz), detail::len(kx), Ninplane, Nz,
                                detail::mptr(dcf)));
  return dcf;
}

// Coil-major images G / (dcf .* data_c) (directRecon.cpp:108-133).
template <typename T1, typename RCol, typename CxCol>
CxCol gridCoilImages(const Gnufft<T1>& G, const RCol& dcf, const CxCol& data, uword Ncoils) {
  CxCol out(G.n_image() * Ncoils);
  check(pg_grid_coil_images(G.handle(), detail::ptr(dcf), reinterpret_cast<const float*>(detail::ptr(data)), Ncoils,
                            reinterpret_cast<float*>(detail::mptr(out))));
  return out;
}

// calcSumOfSquaresImage (directRecon.cpp:63-73): sqrt(sum_c |img_c|).
template <typename T1, typename RCol, typename CxCol>
RCol calcSumOfSquaresImage(const CxCol& coilImages, uword Ncoils) {
  const uword n = detail::len(coilImages) / Ncoils;
  RCol out(n);
  check(pg_sum_of_squares_image(reinterpret_cast<const float*>(detail::ptr(coilImages)), n, Ncoils,
                                detail::mptr(out)));
  return out;
}

// writeNiftiRealImage / writeNiftiMagPhsImage (processNIFTI.hpp:37-117):
// "<filename>.nii", or "<filename>_mag.nii" and "<filename>_phs.nii".
template <typename T1, typename RCol>
void writeNiftiRealImage(const std::string& filename, const RCol& imageData, uword Nx, uword Ny, uword Nz = 1,
                         uword Nslab = 1, uword N_TR = 1) {
  check(pg_write_nifti_real(filename.c_str(), detail::ptr(imageData), Nx, Ny, Nz, Nslab, N_TR));
}
template <typename T1, typename CxCol>
void writeNiftiMagPhsImage(const std::string& filename, const CxCol& imageData, uword Nx, uword Ny, uword Nz,
                           uword Nslab = 1, uword N_TR = 1) {
  check(pg_write_nifti_mag_phs(filename.c_str(), reinterpret_cast<const float*>(detail::ptr(imageData)), Nx, Ny, Nz,
                               Nslab, N_TR));
}

// acqTracking over an in-memory acquisition list (acqTracking.h:14); the
// acquisitions' arrays are borrowed.
class acqTracking {
 public:
  acqTracking(const std::vector<pg_acquisition>& acqs, const pg_encoding_limits& limits) {
    check(pg_acq_index_create(&h_, acqs.data(), acqs.size(), &limits));
  }
  acqTracking(const acqTracking&) = delete;
  acqTracking& operator=(const acqTracking&) = delete;
  ~acqTracking() { pg_acq_index_destroy(h_); }
  pg_acq_index handle() const { return h_; }
  long long acqArray(uword shot, uword par, uword slice, uword rep, uword avg, uword echo, uword phase) const {
    int64_t a = -1;
    check(pg_acq_index_lookup(h_, (uint32_t)shot, (uint32_t)par, (uint32_t)slice, (uint32_t)rep, (uint32_t)avg,
                              (uint32_t)echo, (uint32_t)phase, &a));
    return a;
  }

 private:
  pg_acq_index h_ = nullptr;
};

// getCompleteISMRMRDAcqData (processIsmrmrd.hpp:361-471) over the index.
template <typename T1, typename CxCol, typename RCol>
void getCompleteISMRMRDAcqData(const acqTracking& acqTrack, uword NSlice, uword NRep, uword NAve, uword NEcho,
                               uword NPhase, CxCol& data, RCol& kx, RCol& ky, RCol& kz, RCol& tvec) {
  uint64_t na = 0, nro = 0, nc = 0;
  check(pg_acq_gather_size(acqTrack.handle(), (uint32_t)NSlice, (uint32_t)NRep, (uint32_t)NAve, (uint32_t)NEcho,
                           (uint32_t)NPhase, &na, &nro, &nc));
  data = CxCol(na * nro * nc);
  kx = RCol(na * nro);
  ky = RCol(na * nro);
  kz = RCol(na * nro);
  tvec = RCol(na * nro);
  check(pg_acq_gather(acqTrack.handle(), (uint32_t)NSlice, (uint32_t)NRep, (uint32_t)NAve, (uint32_t)NEcho,
                      (uint32_t)NPhase, reinterpret_cast<float*>(detail::mptr(data)), detail::mptr(kx),
                      detail::mptr(ky), detail::mptr(kz), detail::mptr(tvec)));
}

// The request server (pg_server_*).  The reference has no server: its
// ISMRMRD driver reconstructs one image after another
// (PowerGridIsmrmrd.cpp:191-264).  Here requests are batched, admitted by HBM
// footprint and overlapped on the device; submit(acqTracking, ...) runs that
// driver's whole image loop over an acquisition index.
class Server {
 public:
  Server(uint64_t hbm_budget_bytes, uint32_t max_inflight) {
    const pg_server_config c{hbm_budget_bytes, max_inflight, 0};
    check(pg_server_create(&h_, &c));
  }
  Server(const Server&) = delete;
  Server& operator=(const Server&) = delete;
  ~Server() { pg_server_destroy(h_); }
  // A request's arrays must stay valid until wait() (or poll()) reports it done.
  uint64_t submit(const pg_request& r) {
    uint64_t t = 0;
    check(pg_submit(h_, &r, &t));
    return t;
  }
  uint64_t submit(const acqTracking& acqs, const pg_acq_request& q) {
    uint64_t t = 0;
    check(pg_submit_acquisitions(h_, acqs.handle(), &q, &t));
    return t;
  }
  pg_request_stats wait(uint64_t ticket) {
    pg_request_stats st{};
    check(pg_wait(h_, ticket, &st));
    return st;
  }
  // true (stats filled) once the request is done
  bool poll(uint64_t ticket, pg_request_stats* st) {
    const pg_status s = pg_poll(h_, ticket, st);
    if (s == PG_NOT_READY) return false;
    check(s);
    return true;
  }
  void cancel(uint64_t ticket) { check(pg_cancel(h_, ticket)); }

 private:
  pg_server h_ = nullptr;
};

template <typename T1>
struct QuadPenalty {
  pg_penalty p;
  QuadPenalty(uword nx, uword ny, uword nz, T1 beta, uword dims2penalize = 3)
      : p{PG_PENALTY_QUAD, nx, ny, nz, (float)beta, 1.0f, dims2penalize} {}
};

template <typename T1>
struct TVPenalty {
  pg_penalty p;
  TVPenalty(uword nx, uword ny, uword nz, T1 beta, T1 delta, uword dims2penalize = 3)
      : p{PG_PENALTY_TV, nx, ny, nz, (float)beta, (float)delta, dims2penalize} {}
};

// R_lowRank(R1, rank, nImages, vBasis) (lowRank/R_lowRank.h:52): R1 applied
// to the columns of X * vBasis^H.  vBasis is rank x nImages; as in the
// reference, a solve needs rank == nImages.
template <typename T1, typename Robj>
struct R_lowRank {
  pg_penalty p;
  uword Nrank, Nimg;
  std::vector<std::complex<float>> v;
  template <typename CxMat>
  R_lowRank(const Robj& R1, uword rank, uword nImages, const CxMat& vBasis)
      : p(R1.p), Nrank(rank), Nimg(nImages),
        v(reinterpret_cast<const std::complex<float>*>(detail::ptr(vBasis)),
          reinterpret_cast<const std::complex<float>*>(detail::ptr(vBasis)) + rank * nImages) {}
};

namespace detail {
template <typename R>
struct is_lowrank : std::false_type {};
template <typename T1, typename Robj>
struct is_lowrank<R_lowRank<T1, Robj>> : std::true_type {};
}  // namespace detail

// solve_pwls_pcg(xInitial, A, W, yi, R, niter) on the device (a QuadPenalty,
// TVPenalty or R_lowRank R).
template <typename T1, typename Tobj, typename Robj, typename CxCol, typename RCol>
CxCol solve_pwls_pcg(const CxCol& xInitial, const Tobj& A, const RCol& W, const CxCol& yi, const Robj& R,
                     uword niter) {
  CxCol x(A.n_image());
  uint64_t done = 0;
  if constexpr (detail::is_lowrank<Robj>::value) {
    check(pg_pcg_solve_lowrank(A.handle(), reinterpret_cast<const float*>(detail::ptr(xInitial)), detail::ptr(W),
                               reinterpret_cast<const float*>(detail::ptr(yi)), &R.p, R.Nrank, R.Nimg,
                               reinterpret_cast<const float*>(R.v.data()), niter,
                               reinterpret_cast<float*>(detail::mptr(x)), &done));
  } else {
    check(pg_pcg_solve(A.handle(), reinterpret_cast<const float*>(detail::ptr(xInitial)), detail::ptr(W),
                       reinterpret_cast<const float*>(detail::ptr(yi)), &R.p, niter,
                       reinterpret_cast<float*>(detail::mptr(x)), &done));
  }
  return x;
}

// reconSolve(data, Sg, R, kx, ky, kz, Nx, Ny, Nz, tvec, niter): W = 1, x0 = 0.
template <typename T1, typename TObj, typename RObj, typename CxCol, typename RCol>
CxCol reconSolve(const CxCol& data, TObj& Sg, RObj R, const RCol&, const RCol&, const RCol&, uword, uword, uword,
                 const RCol&, uword niter) {
  CxCol x(Sg.n_image());
  check(pg_recon_solve(Sg.handle(), &R.p, reinterpret_cast<const float*>(detail::ptr(data)), niter,
                       reinterpret_cast<float*>(detail::mptr(x))));
  return x;
}

}  // namespace pg
