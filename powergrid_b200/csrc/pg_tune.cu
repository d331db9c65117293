// Autotuner for the gridding parameters: tile edge and bin size (samples per
// subproblem) of the sample binning, and the coils per block of the spread
// and gather kernels.
//
// Candidates are timed with CUDA events on the operator's own stream and
// plan (forward + adjoint over a batch of up to 4 coils with synthetic
// values), in two rounds: tile x bin size with the default coils per block,
// then the coils per block for the winning binning.  Results are cached per
// problem shape (dimension, image and sample counts, segments, window, coil
// batch; the sample count by its power-of-two bucket), so operators of a
// recurring shape are tuned once per process.  Callers that cannot afford a
// search (the request server) only take cached results.
// PG_AUTOTUNE=0 keeps the defaults (and the PG_TILE2D ... overrides);
// PG_TUNE_LOG=1 prints each search's choice to stderr.
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "pg_nufft.cuh"

namespace pg {
namespace {

// Problem shape; the sample count enters as its power-of-two bucket, so
// trajectories of similar length share a tuning.
struct TuneKey {
  int dim, nx, ny, nz, mlog, L, K, C;
  bool operator<(const TuneKey& o) const {
    return std::tie(dim, nx, ny, nz, mlog, L, K, C) < std::tie(o.dim, o.nx, o.ny, o.nz, o.mlog, o.L, o.K, o.C);
  }
};
int log2_bucket(uint64_t v) {
  int b = 0;
  while ((2ull << b) <= v) ++b;
  return b;
}
std::mutex g_tune_mu;
std::map<TuneKey, NufftTune> g_tuned;

bool tuning_enabled() {
  const char* e = getenv("PG_AUTOTUNE");
  return !(e && e[0] == '0');
}

__global__ void k_fill_pattern(uint64_t n, float2* __restrict__ v) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = make_float2(1.f + (float)(i % 7) * 0.125f, 0.5f - (float)(i % 5) * 0.25f);
}

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() { cudaEventCreate(&a); cudaEventCreate(&b); }
  ~Timer() { cudaEventDestroy(a); cudaEventDestroy(b); }
};

// Milliseconds of `reps` applications (after one untimed one); huge on error.
template <typename F>
float time_ms(F&& f, cudaStream_t s, int reps) {
  if (f() != PG_OK) return 1e30f;
  Timer t;
  cudaEventRecord(t.a, s);
  for (int r = 0; r < reps; ++r)
    if (f() != PG_OK) return 1e30f;
  cudaEventRecord(t.b, s);
  if (cudaEventSynchronize(t.b) != cudaSuccess) { cudaGetLastError(); return 1e30f; }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t.a, t.b);
  return ms;
}

// Timed applications per coils-per-block candidate: the spread's choices
// differ by ~3 % at the configurations' sizes, below the spread of 2 runs.
constexpr int kCoilReps = 8;

}  // namespace

pg_status nufft_autotune(NufftPlan* p, int L, int K, const int* l0_host, const float2* aa_host, int C,
                         std::unique_ptr<Binning>* bin, bool search, cudaStream_t s) {
  const NufftGeom& g = p->g;
  const int Ct = std::max(1, std::min(C, 4));
  const TuneKey key{g.dim, g.Nx, g.Ny, g.Nz, log2_bucket(p->M), L, K, Ct};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      const NufftTune& t = it->second;
      const bool rebin = (g.dim == 2 ? t.tile2d != p->tune.tile2d : t.tile3d != p->tune.tile3d) ||
                         (g.dim == 2 ? t.submax2d != p->tune.submax2d : t.submax3d != p->tune.submax3d);
      p->tune = t;
      if (rebin || !*bin) return nufft_build_binning(p, L, K, l0_host, aa_host, bin, s);
      return PG_OK;
    }
  }
  if (!search || !tuning_enabled()) {
    if (!*bin) return nufft_build_binning(p, L, K, l0_host, aa_host, bin, s);
    return PG_OK;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cs);
  if (cs != cudaStreamCaptureStatusNone) {   // no timing inside a capture
    if (!*bin) return nufft_build_binning(p, L, K, l0_host, aa_host, bin, s);
    return PG_OK;
  }

  const uint64_t N = g.nimg(), M = p->M;
  DevBuf<float2> x, y;
  PG_TRY(x.alloc(N));
  PG_TRY(y.alloc(M * (uint64_t)Ct));
  PG_LAUNCH(k_fill_pattern, ceil_div(N, 256), 256, 0, s, N, x.p);
  PG_LAUNCH(k_fill_pattern, ceil_div(M * (uint64_t)Ct, 256), 256, 0, s, M * (uint64_t)Ct, y.p);

  const NufftTune base = p->tune;
  std::vector<int> tiles = (g.dim == 2) ? std::vector<int>{16, 32} : std::vector<int>{8};
  const std::vector<int> submaxes = {128, 256, 512};
  NufftTune best = base;
  std::unique_ptr<Binning> best_bin;
  float best_ms = 3e30f;
  for (int tile : tiles)
    for (int sm : submaxes) {
      NufftTune t = base;
      if (g.dim == 2) { t.tile2d = tile; t.submax2d = sm; } else { t.tile3d = tile; t.submax3d = sm; }
      p->tune = t;
      std::unique_ptr<Binning> cand;
      PG_TRY(nufft_build_binning(p, L, K, l0_host, aa_host, &cand, s));
      NufftBatch b;
      b.C = Ct;
      b.bin = cand.get();
      b.data_stride = M;
      const float ms = time_ms([&] {
        pg_status st = nufft_forward(p, b, x.p, y.p, s);
        return st == PG_OK ? nufft_adjoint(p, b, y.p, x.p, s) : st;
      }, s, 2);
      if (ms < best_ms) { best_ms = ms; best = t; best_bin = std::move(cand); }
    }
  if (!best_bin) return set_error(PG_CUDA_ERROR, "autotune: no candidate ran");
  p->tune = best;
  NufftBatch b;
  b.C = Ct;
  b.bin = best_bin.get();
  b.data_stride = M;
  if (Ct > 1) {
    float bs = 3e30f, bg = 3e30f;
    int cs_best = best.spread_cc, cg_best = best.gather_cc;
    for (int cc : {1, 2, 4}) {
      if (cc > Ct) break;
      p->tune.spread_cc = cc;
      const float ms = time_ms([&] { return nufft_adjoint(p, b, y.p, x.p, s); }, s, kCoilReps);
      if (ms < bs) { bs = ms; cs_best = cc; }
    }
    p->tune.spread_cc = cs_best;
    for (int cc : {1, 2, 4}) {
      if (cc > Ct) break;
      p->tune.gather_cc = cc;
      const float ms = time_ms([&] { return nufft_forward(p, b, x.p, y.p, s); }, s, kCoilReps);
      if (ms < bg) { bg = ms; cg_best = cc; }
    }
    p->tune.gather_cc = cg_best;
  }
  PG_CUDA(cudaStreamSynchronize(s));
  *bin = std::move(best_bin);
  if (const char* e = getenv("PG_TUNE_LOG"); e && e[0] == '1')
    std::fprintf(stderr, "powergrid_b200 autotune: %dD %dx%dx%d, M=%llu, L=%d, K=%d, %d coils: tile %d, %d samples "
                 "per subproblem, spread %d / gather %d coils per block\n", g.dim, g.Nx, g.Ny, g.Nz,
                 (unsigned long long)M, L, K, Ct, g.dim == 2 ? p->tune.tile2d : p->tune.tile3d,
                 g.dim == 2 ? p->tune.submax2d : p->tune.submax3d, p->tune.spread_cc, p->tune.gather_cc);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned.emplace(key, p->tune);
  return PG_OK;
}

}  // namespace pg
