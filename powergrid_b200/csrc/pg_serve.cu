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
#include <chrono>
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

struct Ticket {
  uint64_t id = 0;
  std::once_flag shared_once;
  pg_status shared_st = PG_OK;
  std::unique_ptr<SharedPlan> shared;
  pg_request req{};
  uint64_t footprint = 0;        // one slice (admission check at submit)
  uint64_t slices_per_job = 1;
  int jobs_total = 0;
  int jobs_left = 0;
  int jobs_started = 0;
  std::atomic<bool> cancel{false};
  pg_request_stats st{};
  bool done = false;
};

struct Job {
  std::shared_ptr<Ticket> t;
  uint64_t slice = 0;            // first slice
  uint64_t count = 1;            // slices
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

  // The request's shared part, built by its first job (the others wait).
  static pg_status build_shared(Ticket& T, cudaStream_t s) {
    const pg_request& r = T.req;
    const uint64_t N = r.nx * r.ny * r.nz, M = r.n_samples;
    auto sp = std::make_unique<SharedPlan>();
    PG_TRY(arena_open(&sp->arena, shared_footprint(r), s));
    arena_install(&sp->arena);
    pg_status st = make_gnufft(&sp->G, M, 2.0f, r.nx, r.ny, r.nz, r.kx, r.ky, r.kz, s);
    if (st == PG_OK) st = make_timeseg(&sp->A, sp->G.get(), r.field_map, r.t, M, N, r.L, 1, 1, s);
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
    const pg_request& r = j.t->req;
    const uint64_t N = r.nx * r.ny * r.nz, M = r.n_samples, C = r.nc;
    const uint64_t sl = j.slice, ns = j.count;
    const double t0 = now_ms();
    double t1 = t0;
    Ticket& T = *j.t;
    std::call_once(T.shared_once, [&] { T.shared_st = build_shared(T, s); });
    if (T.shared_st != PG_OK) return T.shared_st;
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
        st = make_gnufft_shared(&G, *T.shared->G);
        if (st != PG_OK) break;
        G->plan->budget_bytes = kJobGridBytes;
        // the job's slices as one operator: their coils share every gridding launch
        st = make_slice_batch(&A, G.get(), T.shared->A.get(), ns, C, r.field_map + sl * N,
                              r.sense_map + 2 * sl * N * C, s);
        if (st != PG_OK) break;
        st = y.upload(reinterpret_cast<const float2*>(r.data) + sl * M * C, ns * M * C, s);
        if (st != PG_OK) break;
        if ((st = x.alloc(ns * N)) != PG_OK) break;
        if ((st = it.alloc(ns)) != PG_OK) break;
        pg_penalty R{PG_PENALTY_QUAD, r.nx, r.ny, r.nz, r.beta, 1.0f, 3};
        t1 = now_ms();
        // one PCG over the stack, inner products and steps per slice
        st = pcg_solve_device(A.get(), nullptr, nullptr, y.p, R, r.niter, x.p, it.p, s, &j.t->cancel);
        if (st != PG_OK) break;
        cudaError_t e = cudaMemcpyAsync(r.image_out + 2 * sl * N, x.p, ns * N * sizeof(float2), cudaMemcpyDeviceToHost,
                                        s);
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
      if (st != PG_OK && st != PG_CANCELLED && log_errors)
        std::fprintf(stderr, "powergrid_b200 server: request %llu slices %llu-%llu: %s\n",
                     (unsigned long long)job.t->id, (unsigned long long)job.slice,
                     (unsigned long long)(job.slice + job.count - 1), pg_last_error());
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
          std::snprintf(t.st.error, sizeof(t.st.error), "slices %llu-%llu: %s", (unsigned long long)job.slice,
                        (unsigned long long)(job.slice + job.count - 1), pg_last_error());
        }
        if (--t.jobs_left == 0) {
          t.st.t_done_ms = now_ms();
          if (t.cancel.load() && t.st.status == PG_OK) t.st.status = PG_CANCELLED;
          done_shared = std::move(t.shared);
          t.done = true;
          cv_done.notify_all();
        }
      }
      // every job of the request has synchronised its stream
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
      if (--t.jobs_left == 0) { t.done = true; t.st.t_done_ms = now_ms(); }
    }
    sv->pending.clear();
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  for (auto& w : sv->workers) w.join();
  // shared plans of cancelled requests: their builders' streams are gone
  for (auto& kv : sv->tickets)
    if (kv.second->shared) kv.second->shared->arena.stream = default_stream();
  delete sv;
  return PG_OK;
}

pg_status pg_submit(pg_server sv, const pg_request* r, uint64_t* ticket) {
  if (!sv || !r || !ticket) return set_error(PG_INVALID_ARG, "submit: null argument");
  if (!r->kx || !r->ky || !r->t || !r->field_map || !r->sense_map || !r->data || !r->image_out)
    return set_error(PG_INVALID_ARG, "submit: null array");
  if (r->nz > 1 && !r->kz) return set_error(PG_INVALID_ARG, "submit: kz required for 3-D");
  if (r->nx == 0 || r->ny == 0 || r->nz == 0 || r->nc == 0 || r->n_samples == 0)
    return set_error(PG_INVALID_ARG, "submit: empty request");
  auto t = std::make_shared<Ticket>();
  t->req = *r;
  if (t->req.n_slices == 0) t->req.n_slices = 1;
  t->footprint = request_footprint(t->req);
  t->st.bytes_resident = t->footprint;
  t->st.status = PG_OK;
  if (t->footprint > sv->cfg.hbm_budget_bytes)
    return set_error(PG_REJECTED, "request needs %llu bytes per slice, budget is %llu",
                     (unsigned long long)t->footprint, (unsigned long long)sv->cfg.hbm_budget_bytes);
  // slices per job: all of the request's, or as many as fit the budget
  uint64_t k = t->req.n_slices;
  while (k > 1 && job_footprint(t->req, k) > sv->cfg.hbm_budget_bytes) k = (k + 1) / 2;
  t->slices_per_job = k;
  t->jobs_total = t->jobs_left = (int)((t->req.n_slices + k - 1) / k);
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) return set_error(PG_CANCELLED, "server is shutting down");
    t->id = sv->next++;
    t->st.t_submit_ms = now_ms();
    sv->tickets[t->id] = t;
    for (uint64_t sl = 0; sl < t->req.n_slices; sl += k) {
      const uint64_t cnt = std::min<uint64_t>(k, t->req.n_slices - sl);
      sv->pending.push_back(Job{t, sl, cnt, job_footprint(t->req, cnt)});
    }
    *ticket = t->id;
  }
  sv->cv_work.notify_all();
  return PG_OK;
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
