// Operator objects behind the pg_op handle.
#pragma once

#include <atomic>
#include <memory>
#include <vector>

#include "pg_gdft.cuh"
#include "pg_interp.cuh"
#include "pg_nufft.cuh"

enum pg_op_kind {
  PG_OP_GNUFFT = 1, PG_OP_GDFT = 2, PG_OP_TIMESEG = 3, PG_OP_SENSE = 4, PG_OP_PCSENSE_TS = 5, PG_OP_PCSENSE = 6,
  PG_OP_LOWRANK = 7
};

// Per-operator PWLS-PCG state kept between solves (buffers + the captured
// per-iteration graph), defined in pg_pcg.cu.
struct pg_pcg_cache_base {
  virtual ~pg_pcg_cache_base() {}
};

struct pg_op_s {
  int kind = 0;
  std::unique_ptr<pg_pcg_cache_base> pcg_cache;
  uint64_t n_data = 0, n_image = 0;
  // independent problems of equal size stacked in x and y (the PCG solves each
  // with its own scalars); 1 for every operator of the C ABI
  uint64_t n_seg = 1;
  // staging for the host-buffer entry points (kept between calls)
  pg::DevBuf<float2> hx, hy, hx0;
  pg::DevBuf<float> hw;
  pg::DevBuf<uint32_t> hit;
  virtual ~pg_op_s() {}
  virtual pg_status forward(const float2* x, float2* y, cudaStream_t s) = 0;
  virtual pg_status adjoint(const float2* y, float2* x, cudaStream_t s) = 0;
  // Device bytes held by the operator (admission accounting).
  virtual uint64_t resident_bytes() const { return 0; }
};

namespace pg {

// Time-segmentation tables built on the host with the reference's operand
// types (TimeSegmentation.cpp:59-93, 213-218).
struct TsTables {
  int L = 1;
  float tau = 0.f, tmin = 0.f;
  int K = 1;
  std::vector<float2> AA;       // n1 x L (column l contiguous) — full table
  std::vector<int> l0;          // per sample window start
  std::vector<float2> aa_win;   // per sample K values
};
// Segment phases Wo / WoH (L x n2) on the device.
pg_status build_ts_phases(const TsTables& T, const float* field_map, uint64_t n2, DevBuf<float2>* Wo,
                          DevBuf<float2>* WoH, cudaStream_t s);
pg_status build_ts_tables(const float* field_map, const float* tvec, uint64_t n1, uint64_t n2, uint64_t L,
                          uint64_t interptype, uint64_t shots, TsTables* out);
// Interpolator tables AA (none x L, column l contiguous) for one shot's times
// tv (already shifted by T_min), pg_tsinterp.cu.
pg_status ts_aa_minmax(const float* fm, uint64_t n2, const std::vector<float>& tv, int L, float tau,
                       std::vector<float2>* aa);
pg_status ts_aa_histogram(const float* fm, uint64_t n2, const std::vector<float>& tv, int L, float tau,
                          std::vector<float2>* aa);
// Whether the fused gridding can apply a segment window of K segments.
bool segment_window_fits(const NufftPlan& p, int K);

struct GnufftOp : pg_op_s {
  std::unique_ptr<NufftPlan> plan;           // null when gridos != 2 (spatial interpolation only)
  std::unique_ptr<InterpPlan> interp;        // spatial-interpolation tables (Gnufft.cpp:213-337)
  pg_status forward(const float2* x, float2* y, cudaStream_t s) override;
  pg_status adjoint(const float2* y, float2* x, cudaStream_t s) override;
  uint64_t resident_bytes() const override;
};

struct GdftOp : pg_op_s {
  std::unique_ptr<GdftPlan> plan;
  pg_status forward(const float2* x, float2* y, cudaStream_t s) override;
  pg_status adjoint(const float2* y, float2* x, cudaStream_t s) override;
};

struct TimeSegOp : pg_op_s {
  pg_op_s* inner = nullptr;  // not owned (TimeSegmentation.cpp:53)
  TsTables tab;
  DevBuf<float2> Wo, WoH, AAfull;
  std::unique_ptr<Binning> bin;  // when inner is Gnufft
  DevBuf<float2> tmp_img, tmp_data, acc;
  pg_status forward(const float2* x, float2* y, cudaStream_t s) override;
  pg_status adjoint(const float2* y, float2* x, cudaStream_t s) override;
};

struct SenseOp : pg_op_s {
  pg_op_s* inner = nullptr;  // not owned (SENSE.cpp:39)
  uint64_t nc = 0;
  DevBuf<float2> S;
  DevBuf<float2> tmp_img, acc;
  pg_status forward(const float2* x, float2* y, cudaStream_t s) override;
  pg_status adjoint(const float2* y, float2* x, cudaStream_t s) override;
};

struct PcSenseTsOp : pg_op_s {
  uint64_t Ni = 0, Nc = 0, Ns = 0, Nd = 0;
  std::vector<std::unique_ptr<NufftPlan>> plans;
  std::vector<std::unique_ptr<Binning>> bins;
  std::vector<TsTables> tabs;
  std::vector<DevBuf<float2>> Wo, WoH;
  DevBuf<float2> S, E;
  pg_status forward(const float2* x, float2* y, cudaStream_t s) override;
  pg_status adjoint(const float2* y, float2* x, cudaStream_t s) override;
  uint64_t resident_bytes() const override;
};

// pcSENSE over Gdft (pcSENSE.cpp:40-153): per shot its own Gdft on that shot's
// samples and times, all over one voxel table.
struct PcSenseOp : pg_op_s {
  uint64_t Ni = 0, Nc = 0, Ns = 0, Nd = 0;
  std::vector<std::unique_ptr<GdftPlan>> plans;
  DevBuf<float2> S;     // Ni x Nc coil maps
  DevBuf<float2> E;     // Ni x Ns: conj(exp(-i P_s)) = exp(+i P_s) (pcSENSE.cpp:103)
  DevBuf<float2> tmp;
  pg_status forward(const float2* x, float2* y, cudaStream_t s) override;
  pg_status adjoint(const float2* y, float2* x, cudaStream_t s) override;
  uint64_t resident_bytes() const override;
};

// LRobj (lowRank/LRobj.cpp:27-68): x = vec(X), X N x K; forward sends the
// columns of X v (v: K x Nimg) through the per-image operators, adjoint
// applies their adjoints and multiplies the N x Nimg stack by v^H.  The
// per-image operators are borrowed (the reference holds raw pointers).
struct LowRankOp : pg_op_s {
  uint64_t N = 0, Nd = 0, K = 0, Ni = 0;
  std::vector<pg_op_s*> ops;
  DevBuf<float2> cf;      // Nimg x K: cf[i + Nimg k] = v[k + K i]
  DevBuf<float2> ca;      // K x Nimg: ca[k + K i] = conj(v[k + K i])
  DevBuf<float2> stack;   // N x Nimg image stack
  pg_status forward(const float2* x, float2* y, cudaStream_t s) override;
  pg_status adjoint(const float2* y, float2* x, cudaStream_t s) override;
  uint64_t resident_bytes() const override;
};

// The slices of a served request as one operator.  The reference's driver
// builds SENSE over TimeSegmentation over Gnufft for each slice and solves them
// one after another (PowerGridIsmrmrd.cpp:191-264); here the ns slices, which
// share the trajectory, the segment windows and the sample binning, are
// stacked, x = [x_0; ...; x_{ns-1}] (N each), y = [y_0; ...] (nc * M each,
// coil-major), and one gridding launch carries every slice's coils (slice s,
// coil c = virtual coil s * nc + c).  n_seg = ns: the PCG solves each slice
// with its own FP64 scalars and early exits.
struct SliceBatchOp : pg_op_s {
  GnufftOp* G = nullptr;            // not owned: the job's plan (own workspace)
  const TimeSegOp* ts = nullptr;    // not owned: segment windows and binning; null when L <= 1
  uint64_t ns = 1, nc = 1, N = 0, M = 0;
  int L = 1;
  DevBuf<float2> S;                 // ns x nc x N coil maps
  DevBuf<float2> Wo, WoH;           // ns x L x N segment phases
  pg_status forward(const float2* x, float2* y, cudaStream_t s) override;
  pg_status adjoint(const float2* y, float2* x, cudaStream_t s) override;
};
// field_maps[sl]: slice sl's field map (N); sense_maps[sl]: its coil maps
// (nc x N complex, interleaved floats).  Host memory, read before return.
pg_status make_slice_batch(std::unique_ptr<SliceBatchOp>* out, GnufftOp* G, const TimeSegOp* ts, uint64_t ns,
                           uint64_t nc, const float* const* field_maps, const float* const* sense_maps,
                           cudaStream_t s);

// out[:, a] = sum_b in[:, b] * C[a + Kout b] over columns of length N, the sum
// in order of b; out is stored column-major N x Kout, or transposed (Kout x N,
// out[a + Kout n]) when transposed_out.
pg_status mix_columns(uint64_t N, int Kin, int Kout, const float2* in, const float2* C, bool transposed_out,
                      float2* out, cudaStream_t s);

pg_status make_gnufft(std::unique_ptr<GnufftOp>* out, uint64_t data_length, float gridos, uint64_t nx, uint64_t ny,
                      uint64_t nz, const float* kx, const float* ky, const float* kz, cudaStream_t s);
pg_status make_timeseg(std::unique_ptr<TimeSegOp>* out, pg_op_s* G, const float* field_map, const float* tvec,
                       uint64_t n1, uint64_t n2, uint64_t L, uint64_t interptype, uint64_t shots, cudaStream_t s);
pg_status make_sense(std::unique_ptr<SenseOp>* out, pg_op_s* G, const float* sense_map, uint64_t n1, uint64_t n2,
                     uint64_t nc, cudaStream_t s);
// Autotune the gridding under G (Gnufft or TimeSegmentation<Gnufft>) for
// batches of nc coils (search = false: cached choices only); no-op for other
// operators.
pg_status tune_for_coils(pg_op_s* G, int nc, bool search, cudaStream_t s);
// Operators that reuse the trajectory tables, time-segment windows and binning
// of existing ones (which must outlive them) and own only their workspaces
// and, for TimeSegmentation, the segment phases of their own field map.
pg_status make_gnufft_shared(std::unique_ptr<GnufftOp>* out, const GnufftOp& src);
pg_status make_timeseg_shared(std::unique_ptr<TimeSegOp>* out, pg_op_s* G, const TimeSegOp& src,
                              const float* field_map, cudaStream_t s);
// Device PWLS-PCG (pg_pcg.cu).  cancel (may be null) is polled between
// iterations.  resume: continue from the solver state on the operator (x0
// ignored) for niter more iterations.
pg_status pcg_solve_device(pg_op_s* A, const float2* x0, const float* W, const float2* y, const pg_penalty& R,
                           uint64_t niter, float2* xout, uint32_t* iters_dev, cudaStream_t s,
                           const std::atomic<bool>* cancel = nullptr, bool resume = false);

}  // namespace pg
