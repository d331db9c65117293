// Gridding NUFFT on sm_100a: the device side of Gnufft (Gnufft.cpp,
// gridding.cpp, griddingSupport.cpp), batched over coils and time segments.
#pragma once

#include <map>
#include <memory>

#include "pg_common.cuh"

namespace pg {

// Oversampled-grid geometry (gridding.cpp:437-446).  Image and grid are
// y-fastest: image p = y + Ny*(x + Nx*z), grid g = gy + Gy*(gx + Gx*gz).
struct NufftGeom {
  int dim = 2;
  int Nx = 1, Ny = 1, Nz = 1;
  int Gx = 1, Gy = 1, Gz = 1;
  float os = 2.f, kw = 4.f, beta = 0.f;
  int nlut = 0;
  // index shifts folded into the kernels (griddingSupport.cpp:372-627)
  int pad_off[3];      // zero_pad offset per axis (x, y, z)
  int crop_off[3];     // crop_center offset per axis
  int fs[3];           // fftshift amount (floor(G/2))
  int ifs[3];          // ifftshift amount (ceil(G/2) in-plane, floor along z)
  float sign_c = 1.f;  // prod over gridded axes of (-1)^(G/2): checkerboard constant
  __host__ __device__ uint64_t nimg() const { return (uint64_t)Nx * Ny * Nz; }
  __host__ __device__ uint64_t ngrid() const { return (uint64_t)Gx * Gy * Gz; }
};

// Adjoint tile shape (grid cells per tile) and its padded shared-memory extent.
struct TileShape {
  int TX, TY, TZ;      // tile size
  int PX, PY, PZ;      // padded smem extent (>= T + 8 along gridded axes)
  int ntx, nty, ntz;   // tiles per axis
};

// Tunable gridding parameters (tile edge, samples per subproblem, coils per
// block).  Defaults can be overridden with PG_TILE2D, PG_TILE3D, PG_SUBMAX2D,
// PG_SUBMAX3D, PG_SPREAD_CC, PG_GATHER_CC.
struct NufftTune {
  int tile2d = 16, tile3d = 8;        // measured best on cfg2 (B200): 16 > 32 > 64
  int submax2d = 256, submax3d = 256;
  int spread_cc = 2, gather_cc = 2;
  static NufftTune defaults();
};

// Per-(trajectory, segmentation) sample binning used by both directions.
// All per-sample arrays are in sorted order (stable by bin key).
struct Binning {
  int K = 1;                 // segment-window length per sample
  int L = 1;                 // segments
  uint64_t M = 0;            // samples
  TileShape tile{};
  DevBuf<uint32_t> perm;     // sorted -> original sample index
  DevBuf<uint2> start;       // (sx | sy << 16, sz): first of 8 taps per axis
  DevBuf<float> wxy;         // 16 per sample: wx[8], wy[8]
  DevBuf<float> wz;          // 8 per sample (3-D)
  DevBuf<int> l0;            // segment-window start per sample
  DevBuf<float2> aa;         // K per sample: interpolator values AA(m, l0..l0+K-1)
  DevBuf<int4> subprob;      // (tile index, l0, first sorted sample, count)
  DevBuf<uint32_t> keys;     // bin key per original sample
  int nsub = 0;
  int submax = 0;            // most samples in one subproblem
  uint64_t nkeys = 0;
};

// Grid workspace and cuFFT work area.  Plans of one geometry that run back
// to back on one stream (the shots of pcSenseTimeSeg) share a single one.
struct NufftWork {
  DevBuf<float2> grids;     // FFT output (forward) / spread target (adjoint, cuFFT path)
  // Spread target of the 2-D adjoint on the plan's own FFT passes.  It is zero
  // at the start of every adjoint: zeroed when allocated, and the first
  // inverse FFT pass zeroes each cell after reading it.  agrids_clean is
  // false from the spread until that pass is enqueued, so an adjoint that
  // stops in between (an error) makes the next one clear it first.
  DevBuf<float2> agrids;
  bool agrids_clean = false;
  DevBuf<float2> fin;       // forward FFT input; its zero-pad border stays zero
  DevBuf<float2> vs;        // adjoint: per-sample segment values in binned order
  DevBuf<float2> rimg;      // adjoint with the plan's own FFT passes: one image per grid
  DevBuf<unsigned> queue;   // work-queue words of the persistent spread launches
  DevBuf<char> fft_work;
};

struct NufftPlan {
  NufftGeom g;
  NufftTune tune;
  uint64_t M = 0;
  DevBuf<float> kx, ky, kz;      // original order
  DevBuf<float> lut;
  float lut_max = 0.f;           // largest per-axis tap weight
  DevBuf<float> deap;            // Nx + Ny + Nz reciprocal-transform factors
  DevBuf<float> deapf;           // per voxel 1/(OS^d k), 0 where k is NaN
  bool own_fft = false;          // pruned fused 2-D FFT passes instead of cuFFT
  DevBuf<float2> tw2d;           // their twiddle table
  std::unique_ptr<Binning> plain;  // binning without segmentation (L = 1)
  // grid workspace (possibly shared) and cuFFT plans, keyed by batch size
  std::shared_ptr<NufftWork> work = std::make_shared<NufftWork>();
  std::map<int, std::pair<cufftHandle, size_t>> ffts;  // batch -> (pooled plan, work bytes)
  size_t budget_bytes = 8ull << 30;  // grid workspace limit per plan
  ~NufftPlan();
};

// What surrounds the gridding in one batched application.
struct NufftBatch {
  int C = 1;                     // coils in this call
  const float2* S = nullptr;     // C x N coil maps (coil-major) or null
  const float2* E = nullptr;     // N extra image factor (shot phase) or null
  const float2* Wo = nullptr;    // L x N segment phases (forward)
  const float2* WoH = nullptr;   // L x N (adjoint)
  const Binning* bin = nullptr;  // segmentation binning (L, K, AA) or plan->plain
  uint64_t data_stride = 0;      // elements between coils in the data vector
  bool accumulate = false;       // adjoint: add into x instead of overwrite
  // Several images in one call (the slices of a request): coil c belongs to
  // image c / cgroup, whose x (forward input,
  // adjoint output) starts image_stride elements after the previous one and
  // whose Wo / WoH set phase_stride elements after the previous one.  S then
  // holds C = images x cgroup coil maps.  0: one image.
  int cgroup = 0;
  uint64_t image_stride = 0, phase_stride = 0;
};

pg_status nufft_plan_create(std::unique_ptr<NufftPlan>* out, uint64_t M, float gridos, int nx, int ny, int nz,
                            const float* kx, const float* ky, const float* kz, cudaStream_t s);
// Binning for a segmentation: l0_host/aa_host (K per sample, original order)
// or null for the unsegmented case.
pg_status nufft_build_binning(NufftPlan* p, int L, int K, const int* l0_host, const float2* aa_host,
                              std::unique_ptr<Binning>* out, cudaStream_t s);
pg_status nufft_plain_binning(NufftPlan* p, cudaStream_t s);
// A plan that reads src's trajectory tables (src must outlive it) and has a
// workspace of its own, so it can run concurrently with src on another stream.
pg_status nufft_plan_share(const NufftPlan& src, std::unique_ptr<NufftPlan>* out);
// A binning that views b's device arrays (b must outlive it).
std::unique_ptr<Binning> binning_share(const Binning& b);
pg_status nufft_forward(NufftPlan* p, const NufftBatch& b, const float2* x, float2* y, cudaStream_t s);
pg_status nufft_adjoint(NufftPlan* p, const NufftBatch& b, const float2* y, float2* x, cudaStream_t s);

// Choose tile edge, bin size and coils per block for a batch of C coils by
// timing candidates on stream s (cached per problem shape; with search =
// false only a cached choice or the defaults), and leave the matching
// binning in *bin (kept if it already matches).  l0_host/aa_host as for
// nufft_build_binning.
pg_status nufft_autotune(NufftPlan* p, int L, int K, const int* l0_host, const float2* aa_host, int C,
                         std::unique_ptr<Binning>* bin, bool search, cudaStream_t s);

// Host copies of the LUT and beta exactly as Gnufft builds them.
void kb_table(float gridos, std::vector<float>* lut, float* beta);

}  // namespace pg
