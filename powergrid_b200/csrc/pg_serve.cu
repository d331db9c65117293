// Request server: continuous batching of time-segmented SENSE reconstructions.
//
// The reference drivers reconstruct one slice/echo/repetition after another
// (PowerGridIsmrmrd.cpp:191-264), each with its own Gnufft, TimeSegmentation,
// SENSE and reconSolve.  Here the slices of a request, which share the
// trajectory, the segment windows and the sample binning, are batched: a job
// is a run of a request's slices (all of them, or as many as fit the HBM
// budget) solved as ONE stacked operator — every gridding launch carries the
// coils of all its slices — and one PCG whose inner products, step sizes and
// early exits are kept per slice (SliceBatchOp, pg_pcg.cu segments), so each
// slice's image is the one its own solve gives.  Jobs are admitted in FIFO
// order whenever a worker slot is free and the summed device footprint of
// resident jobs stays within the budget.  Every worker owns a CUDA stream, so
// admitted jobs overlap on the GPU, and a job that finishes frees its slot and
// memory for the next arrival.  A job keeps its trajectory, maps and PCG state
// resident in a private device arena (stream-ordered pool allocations, no
// cudaMalloc/cudaFree on the hot path) until its images are copied out.
//
// pg_submit_acquisitions runs the reference driver's whole image loop as one
// request: every (slice, phase, contrast, average, repetition) of an
// acquisition index, each gathered as getCompleteISMRMRDAcqData does
// (processIsmrmrd.hpp:361-471) with its slice's field map and coil maps
// (getISMRMRDCompleteFieldMap / getISMRMRDCompleteSENSEMap,
// processIsmrmrd.hpp:196-266).  The images are grouped by trajectory: those
// whose gathered kx, ky, kz and t are identical share one plan and are
// batched like the slices of pg_submit.
#include <chrono>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "pg_ops.cuh"

namespace pg {
namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// What the slices of one request share: the trajectory tables, the
// time-segment windows and the sample binning, built once by the request's
// first job in an arena of their own and released with the request.
struct SharedPlan {
  Arena arena;
  std::unique_ptr<GnufftOp> G;
  std::unique_ptr<TimeSegOp> A;
  // Runs after every job of the request has synchronised its stream.  The
  // arena is returned on arena.stream, which the owner first points at a
  // stream of the releasing thread: the builder's stream may be capturing a
  // graph on another thread by then, and a free enqueued there would join
  // that capture.
  ~SharedPlan() {
    Arena* prev = arena_current();
    arena_install(&arena);
    A.reset();
    G.reset();
    arena_install(prev);
    arena_release(&arena);
  }
};

// Images that share one trajectory: one SharedPlan, batched jobs.  req holds
// the shape, the trajectory and the images' data (n_slices = images);
// fm[k] / sm[k] are image k's field map and coil maps, out[k] its index in the
// request's output.
struct Group {
  pg_request req{};
  std::vector<const float*> fm, sm;
  std::vector<uint64_t> out;
  size_t data_slot = 0;          // acquisition requests: index of the gathered data in Ticket::owned
  std::once_flag shared_once;
  pg_status shared_st = PG_OK;
  std::unique_ptr<SharedPlan> shared;
  int jobs_left = 0;
};

struct Ticket {
  uint64_t id = 0;
  std::vector<std::unique_ptr<Group>> groups;
  float* image_out = nullptr;
  // gathered host arrays of an acquisition request (trajectories, data); a
  // deque, so growing it keeps the earlier vectors' addresses
  std::deque<std::vector<float>> owned;
  uint64_t footprint = 0;        // one image of the largest group (admission check at submit)
  int jobs_total = 0;
  int jobs_left = 0;
  int jobs_started = 0;
  std::atomic<bool> cancel{false};
  pg_request_stats st{};
  bool done = false;
};

struct Job {
  std::shared_ptr<Ticket> t;
  Group* g = nullptr;
  uint64_t first = 0;            // first image of the group
  uint64_t count = 1;            // images
  uint64_t footprint = 0;
};

uint64_t grid_cells(const pg_request& r) {
  const uint64_t gx = 2 * r.nx, gy = 2 * r.ny, gz = (r.nz == 1) ? 1 : 2 * r.nz;
  return gx * gy * gz;
}

// Per-job grid workspace cap: keeps one job from monopolising the device.
constexpr uint64_t kJobGridBytes = 2ull << 30;

// Device bytes of a request's shared part (trajectory, binning with its
// temporaries, segment phases of the first slice).
uint64_t shared_footprint(const pg_request& r) {
  const uint64_t M = r.n_samples, N = r.nx * r.ny * r.nz;
  const uint64_t L = r.L <= 1 ? 1 : r.L;
  uint64_t b = 3 * M * 4 + 40000 * 4 + (r.nx + r.ny + r.nz) * 4;
  b += M * 2 * (8 + 64 + 32 + 4) + M * (4 + 4 + 3 * 8) + (M + 4096 * L) * 16;
  // device bin sort: (key, chunk) table (at most 16 M entries), bin starts, keys
  const uint64_t nkeys = (r.nz > 1 ? (r.nx / 4 + 1) * (r.ny / 4 + 1) * (r.nz / 4 + 1)
                                   : (r.nx / 8 + 1) * (r.ny / 8 + 1)) * L;
  b += std::min<uint64_t>(nkeys * ((M + 1023) / 1024), 16ull << 20) * 4 + nkeys * 4 + M * 4 + M * 3 * 8;
  b += 3 * L * N * 8;
  return b + b / 4 + (4ull << 20);
}

void release_shared(std::unique_ptr<SharedPlan>& sp) { sp.reset(); }

}  // namespace

// Device bytes of a job of k slices of request r.
uint64_t job_footprint(const pg_request& r, uint64_t k) {
  const uint64_t M = r.n_samples, N = r.nx * r.ny * r.nz, C = r.nc;
  const uint64_t L = r.L <= 1 ? 1 : r.L;
  const uint64_t G = grid_cells(r);
  const bool d3 = r.nz > 1;
  uint64_t b = 0;
  b += 3 * M * 4 + 40000 * 4 + (r.nx + r.ny + r.nz) * 4;          // trajectory, LUT, deapodization
  b += M * (8 + 64 + (d3 ? 32 : 0) + 4 + 4);                        // binning temporaries
  b += M * (4 + 8 + 64 + (d3 ? 32 : 0) + 4 + 3 * 8) + (M / 64 + 4096 * L) * 16;  // binning
  uint64_t grids = k * C * L * G * 8;
  if (grids > kJobGridBytes) grids = std::max<uint64_t>(L * G * 8, (kJobGridBytes / (L * G * 8)) * L * G * 8);
  b += 3 * grids;                                                   // grids, FFT input / adjoint grids, cuFFT work area
  b += k * C * M * 8 * std::min<uint64_t>(L, 3);                    // adjoint segment values (Hanning: K <= 3)
  b += k * (2 * L * N * 8 + C * N * 8);                             // Wo, WoH, coil maps
  b += k * (3 * N * 8 + 3 * C * M * 8 + C * M * 8 + C * M * 4) + 64 * 1024;  // PCG state
  b += k * (C * M * 8 + N * 8);                                     // job input / output
  return b + b / 4 + (32ull << 20);
}

uint64_t request_footprint(const pg_request& r) { return job_footprint(r, 1); }

}  // namespace pg

using namespace pg;

struct pg_server_s {
  pg_server_config cfg{};
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job> pending;
  std::unordered_map<uint64_t, std::shared_ptr<Ticket>> tickets;
  uint64_t used = 0;
  uint32_t running = 0;
  bool stop = false;
  uint64_t next = 1;
  std::vector<std::thread> workers;
  bool log_errors = false;   // PG_SERVE_LOG=1: print failed jobs' messages to stderr

  bool head_fits() const {
    if (pending.empty()) return false;
    const uint64_t f = pending.front().footprint;
    return used + f <= cfg.hbm_budget_bytes || running == 0;
  }

  // A group's shared part, built by its first job (the others wait).
  static pg_status build_shared(Group& T, cudaStream_t s) {
    const pg_request& r = T.req;
    const uint64_t N = r.nx * r.ny * r.nz, M = r.n_samples;
    auto sp = std::make_unique<SharedPlan>();
    PG_TRY(arena_open(&sp->arena, shared_footprint(r), s));
    arena_install(&sp->arena);
    pg_status st = make_gnufft(&sp->G, M, 2.0f, r.nx, r.ny, r.nz, r.kx, r.ky, r.kz, s);
    // the windows and binning depend on t only; the phases of fm[0] go unused
    if (st == PG_OK) st = make_timeseg(&sp->A, sp->G.get(), T.fm[0], r.t, M, N, r.L, 1, 1, s);
    // a search per request would stall the slots: cached tunings only
    if (st == PG_OK) st = tune_for_coils(sp->A.get(), (int)r.nc, false, s);
    if (st == PG_OK) {
      cudaError_t e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) { cudaGetLastError(); st = set_error(PG_CUDA_ERROR, "shared plan: %s", cudaGetErrorString(e)); }
    }
    arena_install(nullptr);
    T.shared = std::move(sp);
    if (st != PG_OK) release_shared(T.shared);   // arena.stream is this thread's stream
    return st;
  }

  pg_status run_job(const Job& j, cudaStream_t s, uint64_t* iters, double* setup_ms, double* solve_ms) {
    Group& g = *j.g;
    const pg_request& r = g.req;
    const uint64_t N = r.nx * r.ny * r.nz, M = r.n_samples, C = r.nc;
    const uint64_t sl = j.first, ns = j.count;
    const double t0 = now_ms();
    double t1 = t0;
    std::call_once(g.shared_once, [&] { g.shared_st = build_shared(g, s); });
    if (g.shared_st != PG_OK) return g.shared_st;
    Arena arena;
    PG_TRY(arena_open(&arena, j.footprint, s));
    arena_install(&arena);
    pg_status st = PG_OK;
    {
      std::unique_ptr<GnufftOp> G;
      std::unique_ptr<SliceBatchOp> A;
      DevBuf<float2> y, x;
      DevBuf<uint32_t> it;
      std::vector<uint32_t> n(ns, 0);
      do {
        st = make_gnufft_shared(&G, *g.shared->G);
        if (st != PG_OK) break;
        G->plan->budget_bytes = kJobGridBytes;
        // the job's images as one operator: their coils share every gridding launch
        st = make_slice_batch(&A, G.get(), g.shared->A.get(), ns, C, g.fm.data() + sl, g.sm.data() + sl, s);
        if (st != PG_OK) break;
        st = y.upload(reinterpret_cast<const float2*>(r.data) + sl * M * C, ns * M * C, s);
        if (st != PG_OK) break;
        if ((st = x.alloc(ns * N)) != PG_OK) break;
        if ((st = it.alloc(ns)) != PG_OK) break;
        pg_penalty R{PG_PENALTY_QUAD, r.nx, r.ny, r.nz, r.beta, 1.0f, 3};
        t1 = now_ms();
        // one PCG over the stack, inner products and steps per image
        st = pcg_solve_device(A.get(), nullptr, nullptr, y.p, R, r.niter, x.p, it.p, s, &j.t->cancel);
        if (st != PG_OK) break;
        cudaError_t e = cudaSuccess;
        // images whose output slots are consecutive leave in one copy
        for (uint64_t k = 0; k < ns && e == cudaSuccess;) {
          uint64_t run = 1;
          while (k + run < ns && g.out[sl + k + run] == g.out[sl + k] + run) ++run;
          e = cudaMemcpyAsync(j.t->image_out + 2 * g.out[sl + k] * N, x.p + k * N, run * N * sizeof(float2),
                              cudaMemcpyDeviceToHost, s);
          k += run;
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(n.data(), it.p, ns * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { cudaGetLastError(); st = set_error(PG_CUDA_ERROR, "job copy-out: %s", cudaGetErrorString(e)); break; }
        uint64_t tot = 0;
        for (uint32_t v : n) tot += v;
        *iters = tot;
      } while (0);
      cudaStreamSynchronize(s);
      // operators and buffers release into the arena (no-ops) before it is returned
    }
    arena_install(nullptr);
    arena_release(&arena);
    cudaStreamSynchronize(s);
    if (cudaError_t e = cudaGetLastError())
      if (log_errors) std::fprintf(stderr, "powergrid_b200 server: job teardown: %s\n", cudaGetErrorString(e));
    *setup_ms = t1 - t0;
    *solve_ms = now_ms() - t1;
    return st;
  }

  void worker() {
    cudaSetDevice(device);
    cudaStream_t s = nullptr;
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    for (;;) {
      Job job;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || head_fits(); });
        if (stop) break;
        job = pending.front();
        pending.pop_front();
        used += job.footprint;
        ++running;
        if (job.t->jobs_started++ == 0) job.t->st.t_start_ms = now_ms();
      }
      uint64_t iters = 0;
      double setup_ms = 0, solve_ms = 0;
      std::unique_ptr<SharedPlan> done_shared;
      if (cudaError_t stale = cudaGetLastError())   // never charge a new job with an earlier error
        if (log_errors) std::fprintf(stderr, "powergrid_b200 server: stale error before a job: %s\n",
                                     cudaGetErrorString(stale));
      pg_status st = job.t->cancel.load() ? PG_CANCELLED : run_job(job, s, &iters, &setup_ms, &solve_ms);
      const unsigned long long img0 = job.g->out[job.first], img1 = job.g->out[job.first + job.count - 1];
      if (st != PG_OK && st != PG_CANCELLED && log_errors)
        std::fprintf(stderr, "powergrid_b200 server: request %llu images %llu-%llu: %s\n",
                     (unsigned long long)job.t->id, img0, img1, pg_last_error());
      {
        std::lock_guard<std::mutex> lk(mu);
        used -= job.footprint;
        --running;
        Ticket& t = *job.t;
        t.st.iters_done += iters;
        t.st.setup_ms += setup_ms;
        t.st.solve_ms += solve_ms;
        if (st != PG_OK && t.st.status == PG_OK) {
          t.st.status = st;
          std::snprintf(t.st.error, sizeof(t.st.error), "images %llu-%llu: %s", img0, img1, pg_last_error());
        }
        // the last job of a group releases its shared plan
        if (--job.g->jobs_left == 0) done_shared = std::move(job.g->shared);
        if (--t.jobs_left == 0) {
          t.st.t_done_ms = now_ms();
          if (t.cancel.load() && t.st.status == PG_OK) t.st.status = PG_CANCELLED;
          t.done = true;
          cv_done.notify_all();
        }
      }
      // every job of the group has synchronised its stream
      if (done_shared) done_shared->arena.stream = s;
      release_shared(done_shared);
      if (cudaError_t e = cudaGetLastError())
        if (log_errors) std::fprintf(stderr, "powergrid_b200 server: releasing a request's shared plan: %s\n",
                                     cudaGetErrorString(e));
      cv_work.notify_all();
    }
    if (s) cudaStreamDestroy(s);
  }
};

extern "C" {

uint64_t pg_request_footprint(const pg_request* req) { return req ? request_footprint(*req) : 0; }

pg_status pg_server_create(pg_server* out, const pg_server_config* cfg) {
  if (!out || !cfg) return set_error(PG_INVALID_ARG, "server: null argument");
  if (cfg->max_inflight == 0 || cfg->max_inflight > 64) return set_error(PG_INVALID_ARG, "server: max_inflight in 1..64");
  if (cfg->hbm_budget_bytes == 0) return set_error(PG_INVALID_ARG, "server: zero HBM budget");
  PG_TRY(ensure_init());
  auto* sv = new pg_server_s;
  sv->cfg = *cfg;
  cudaGetDevice(&sv->device);
  if (const char* e = getenv("PG_SERVE_LOG")) sv->log_errors = e[0] == '1';
  for (uint32_t i = 0; i < cfg->max_inflight; ++i) sv->workers.emplace_back([sv] { sv->worker(); });
  *out = sv;
  return PG_OK;
}

pg_status pg_server_destroy(pg_server sv) {
  if (!sv) return PG_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    for (auto& kv : sv->tickets) kv.second->cancel.store(true);
    // queued jobs are dropped; running ones stop at their next iteration
    for (auto& j : sv->pending) {
      Ticket& t = *j.t;
      if (t.st.status == PG_OK) t.st.status = PG_CANCELLED;
      --j.g->jobs_left;
      if (--t.jobs_left == 0) { t.done = true; t.st.t_done_ms = now_ms(); }
    }
    sv->pending.clear();
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  for (auto& w : sv->workers) w.join();
  // shared plans of cancelled requests: their builders' streams are gone
  for (auto& kv : sv->tickets)
    for (auto& g : kv.second->groups)
      if (g->shared) g->shared->arena.stream = default_stream();
  delete sv;
  return PG_OK;
}

namespace {

// Admission of a formed ticket: every group's one-image job must fit the
// budget; each group is split into jobs of as many images as fit.
pg_status enqueue(pg_server sv, const std::shared_ptr<Ticket>& t, uint64_t* ticket) {
  std::vector<uint64_t> per_job(t->groups.size());
  for (size_t gi = 0; gi < t->groups.size(); ++gi) {
    Group& g = *t->groups[gi];
    const uint64_t f = request_footprint(g.req);
    t->footprint = std::max(t->footprint, f);
    if (f > sv->cfg.hbm_budget_bytes)
      return set_error(PG_REJECTED, "request needs %llu bytes per image, budget is %llu", (unsigned long long)f,
                       (unsigned long long)sv->cfg.hbm_budget_bytes);
    // images per job: all of the group's, or as many as fit the budget
    uint64_t k = g.req.n_slices;
    while (k > 1 && job_footprint(g.req, k) > sv->cfg.hbm_budget_bytes) k = (k + 1) / 2;
    per_job[gi] = k;
    g.jobs_left = (int)((g.req.n_slices + k - 1) / k);
    t->jobs_total += g.jobs_left;
  }
  t->jobs_left = t->jobs_total;
  t->st.jobs = (uint64_t)t->jobs_total;
  t->st.bytes_resident = t->footprint;
  t->st.status = PG_OK;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) return set_error(PG_CANCELLED, "server is shutting down");
    t->id = sv->next++;
    t->st.t_submit_ms = now_ms();
    sv->tickets[t->id] = t;
    for (size_t gi = 0; gi < t->groups.size(); ++gi) {
      Group* g = t->groups[gi].get();
      const uint64_t k = per_job[gi];
      for (uint64_t i = 0; i < g->req.n_slices; i += k) {
        const uint64_t cnt = std::min<uint64_t>(k, g->req.n_slices - i);
        sv->pending.push_back(Job{t, g, i, cnt, job_footprint(g->req, cnt)});
      }
    }
    *ticket = t->id;
  }
  sv->cv_work.notify_all();
  return PG_OK;
}

}  // namespace

pg_status pg_submit(pg_server sv, const pg_request* r, uint64_t* ticket) {
  if (!sv || !r || !ticket) return set_error(PG_INVALID_ARG, "submit: null argument");
  if (!r->kx || !r->ky || !r->t || !r->field_map || !r->sense_map || !r->data || !r->image_out)
    return set_error(PG_INVALID_ARG, "submit: null array");
  if (r->nz > 1 && !r->kz) return set_error(PG_INVALID_ARG, "submit: kz required for 3-D");
  if (r->nx == 0 || r->ny == 0 || r->nz == 0 || r->nc == 0 || r->n_samples == 0)
    return set_error(PG_INVALID_ARG, "submit: empty request");
  auto t = std::make_shared<Ticket>();
  t->image_out = r->image_out;
  auto g = std::make_unique<Group>();
  g->req = *r;
  if (g->req.n_slices == 0) g->req.n_slices = 1;
  const uint64_t N = r->nx * r->ny * r->nz;
  for (uint64_t k = 0; k < g->req.n_slices; ++k) {
    g->fm.push_back(r->field_map + k * N);
    g->sm.push_back(r->sense_map + 2 * k * N * r->nc);
    g->out.push_back(k);
  }
  t->groups.push_back(std::move(g));
  return enqueue(sv, t, ticket);
}

pg_status pg_submit_acquisitions(pg_server sv, pg_acq_index ix, const pg_acq_request* q, uint64_t* ticket) {
  if (!sv || !ix || !q || !ticket) return set_error(PG_INVALID_ARG, "submit acquisitions: null argument");
  if (!q->field_map || !q->sense_map || !q->image_out) return set_error(PG_INVALID_ARG, "submit acquisitions: null array");
  if (q->nx == 0 || q->ny == 0 || q->nz == 0) return set_error(PG_INVALID_ARG, "submit acquisitions: empty image");
  pg_encoding_limits lim{};
  PG_TRY(pg_acq_index_limits(ix, &lim));
  const uint64_t N = q->nx * q->ny * q->nz;
  auto t = std::make_shared<Ticket>();
  t->image_out = q->image_out;
  uint64_t nc = 0, k = 0;
  std::vector<float> d, kx, ky, kz, tv;
  // the reference driver's loop order (PowerGridIsmrmrd.cpp:191-196): slice,
  // phase, contrast, average, repetition (innermost)
  for (uint32_t sl = 0; sl < lim.slices; ++sl)
    for (uint32_t ph = 0; ph < lim.phases; ++ph)
      for (uint32_t ec = 0; ec < lim.contrasts; ++ec)
        for (uint32_t av = 0; av < lim.averages; ++av)
          for (uint32_t rp = 0; rp < lim.repetitions; ++rp, ++k) {
            uint64_t na = 0, nro = 0, nch = 0;
            PG_TRY(pg_acq_gather_size(ix, sl, rp, av, ec, ph, &na, &nro, &nch));
            if (na == 0 || nro == 0)
              return set_error(PG_INVALID_ARG, "submit acquisitions: image %llu (slice %u, repetition %u, average %u, "
                               "contrast %u, phase %u) has no acquisitions", (unsigned long long)k, sl, rp, av, ec, ph);
            if (k == 0) nc = nch;
            if (nch != nc)
              return set_error(PG_INVALID_ARG, "submit acquisitions: image %llu has %llu channels, the first %llu",
                               (unsigned long long)k, (unsigned long long)nch, (unsigned long long)nc);
            const uint64_t M = na * nro;
            d.resize(2 * nc * M);
            kx.resize(M); ky.resize(M); kz.resize(M); tv.resize(M);
            PG_TRY(pg_acq_gather(ix, sl, rp, av, ec, ph, d.data(), kx.data(), ky.data(), kz.data(), tv.data()));
            Group* g = nullptr;
            for (auto& c : t->groups) {
              const pg_request& r = c->req;
              if (r.n_samples == M && !std::memcmp(r.kx, kx.data(), M * 4) && !std::memcmp(r.ky, ky.data(), M * 4) &&
                  !std::memcmp(r.kz, kz.data(), M * 4) && !std::memcmp(r.t, tv.data(), M * 4)) {
                g = c.get();
                break;
              }
            }
            if (!g) {
              auto ng = std::make_unique<Group>();
              g = ng.get();
              t->owned.push_back(kx);
              t->owned.push_back(ky);
              t->owned.push_back(kz);
              t->owned.push_back(tv);
              const size_t o = t->owned.size();
              float tmin = tv[0], tmax = tv[0];
              for (float v : tv) { tmin = std::min(tmin, v); tmax = std::max(tmax, v); }
              // TimeSegments not given: L = ceil((max(t) - min(t)) / 2 ms) for
              // Hanning interpolation (PowerGridIsmrmrd.cpp:217-222)
              const uint64_t L = q->L ? q->L : (uint64_t)std::ceil((double)(tmax - tmin) / 2E-3);
              ng->req = pg_request{q->nx, q->ny, q->nz, 0, nc, M, L, q->niter, q->beta, t->owned[o - 4].data(),
                                   t->owned[o - 3].data(), t->owned[o - 2].data(), t->owned[o - 1].data(),
                                   q->field_map, q->sense_map, nullptr, q->image_out};
              t->owned.emplace_back();   // the group's data, appended image by image
              ng->data_slot = t->owned.size() - 1;
              t->groups.push_back(std::move(ng));
            }
            auto& gd = t->owned[g->data_slot];
            gd.insert(gd.end(), d.begin(), d.end());
            g->fm.push_back(q->field_map + (uint64_t)sl * N);
            g->sm.push_back(q->sense_map + 2 * (uint64_t)sl * N * nc);
            g->out.push_back(k);
            g->req.n_slices++;
          }
  // the data vectors are complete: their addresses are final
  for (auto& g : t->groups) g->req.data = t->owned[g->data_slot].data();
  return enqueue(sv, t, ticket);
}

pg_status pg_poll(pg_server sv, uint64_t ticket, pg_request_stats* stats) {
  if (!sv) return set_error(PG_INVALID_ARG, "poll: null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->tickets.find(ticket);
  if (it == sv->tickets.end()) return set_error(PG_INVALID_ARG, "poll: unknown ticket %llu", (unsigned long long)ticket);
  if (!it->second->done) return PG_NOT_READY;
  if (stats) *stats = it->second->st;
  return PG_OK;
}

pg_status pg_wait(pg_server sv, uint64_t ticket, pg_request_stats* stats) {
  if (!sv) return set_error(PG_INVALID_ARG, "wait: null server");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->tickets.find(ticket);
  if (it == sv->tickets.end()) return set_error(PG_INVALID_ARG, "wait: unknown ticket %llu", (unsigned long long)ticket);
  auto t = it->second;
  sv->cv_done.wait(lk, [&] { return t->done; });
  if (stats) *stats = t->st;
  return PG_OK;
}

pg_status pg_cancel(pg_server sv, uint64_t ticket) {
  if (!sv) return set_error(PG_INVALID_ARG, "cancel: null server");
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->tickets.find(ticket);
    if (it == sv->tickets.end()) return set_error(PG_INVALID_ARG, "cancel: unknown ticket %llu", (unsigned long long)ticket);
    auto t = it->second;
    t->cancel.store(true);
    // drop this request's queued jobs; running ones stop at their next iteration
    for (auto i = sv->pending.begin(); i != sv->pending.end();) {
      if (i->t == t) {
        --i->g->jobs_left;
        if (--t->jobs_left == 0) { t->done = true; t->st.t_done_ms = now_ms(); }
        i = sv->pending.erase(i);
      } else {
        ++i;
      }
    }
    t->st.status = PG_CANCELLED;
  }
  sv->cv_done.notify_all();
  sv->cv_work.notify_all();
  return PG_OK;
}

}  // extern "C"
