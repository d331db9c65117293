"""Benchmark: PCG iterations/s of the 2-D field-corrected SENSE reconstruction.

Workload (one "step" = one full reconstruction): SENSE<TimeSegmentation<Gnufft>>,
128x128 image, L = 8 Hanning segments, 4 coils, 16-interleave spiral with
8192 samples per interleave (131072 samples), 20 ms readout, +-100 Hz field
map, QuadPenalty beta = 1e-3, 20 PWLS-PCG iterations (reconSolve semantics:
W = 1, x0 = 0).  Seeded synthetic inputs stand in for ISMRMRD data.

  value      PCG iterations/s with inputs resident in HBM (device-timed,
             CUDA events per step, L2 flushed between steps, max over ranks)
  e2e        the same metric through the C ABI's host-buffer entry point
             pg_pcg_solve (H2D of the coil data and D2H of the image inside
             the timed region)
  roofline   the adjoint gridding (the grids' clearing and the spread
             kernel, as the reference's gridding_adjoint), timed by a CUDA
             event pair around it in the last PCG iteration of every timed
             step (an instrumented copy of the iteration graph; the other
             iterations replay the plain one), against the measured HBM
             bandwidth; the other stages are timed on extra steps
  cpu_baseline  the reference CPU path on this host's cores (rank 0, N=1)

`--impl reference` times the reference's own CPU implementation of the path
(oracle/_ref when built from the reference sources, else the oracle port).
Multi-GPU: independent replicas (weak scaling), one process per GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

METRIC = "PCG iters/s"
UNIT = "iter/s"
NITER = 20
WORKLOAD = ("SENSE<TimeSegmentation<Gnufft>> 128x128, L=8 Hanning, 4 coils, 16x8192 spiral "
            "(131072 samples/coil), 20 ms readout, +-100 Hz, QuadPenalty beta=1e-3, 20 PCG iterations")


def _config(extra=None):
    c = {"workload": WORKLOAD, "image": [128, 128, 1], "coils": 4, "segments": 8, "samples_per_coil": 131072,
         "pcg_iterations_per_step": NITER, "l2": "flushed between steps (256 MiB write)",
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                v = [s.strip() for s in out.stdout.strip().split(",")]
                if len(v) == 7:
                    self.rows.append(v)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(self.rows[0][1]), "reasons": reasons,
                "samples": len(self.rows)}


def _dist():
    from powergrid_b200.replicas import rank_layout
    return rank_layout()


def _problem():
    from powergrid_b200 import synthetic as S
    return S.config2()


# --------------------------------------------------------------------------------------------
# CPU baseline: the reference CPU path (reference kernels when built, else the oracle port)
# --------------------------------------------------------------------------------------------
def cpu_reference_rate(p, y, iters: int, threads: int):
    """One reconstruction on the reference CPU path (the reference's compiled
    Gnufft kernels when built, else the oracle port): rate, kind, iterations,
    seconds and the image."""
    import oracle as O
    kind = "port"
    if O.reference_available():
        O.use_reference(True)
        kind = "reference"
    O.set_threads(threads)
    op = O.build_problem_op(p, 0)
    t0 = time.perf_counter()
    x, n = op.pcg(y, "quad", p.nx, p.ny, p.nz, p.beta, niter=iters)
    dt = time.perf_counter() - t0
    O.set_threads(1)
    if kind == "reference":
        O.use_reference(False)
    return n / dt, kind, n, dt, x


REFERENCE_IMPL = ("reference kernels (gridding.cpp, griddingSupport.cpp, ftCpu.cpp, fftCPU.cpp) compiled from "
                  "the reference sources; Armadillo layers restated; project FFT behind the FFTW API")


def run_reference_arm(args):
    """The reference CPU path on this host's cores: each step one full
    reconstruction of the workload (the forward of x0 = 0, then NITER PCG
    iterations), timed on the host clock."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    p = _problem()
    import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    y = O.build_problem_op(p, 0).forward(p.x_true)
    for _ in range(args.warmup):
        cpu_reference_rate(p, y, NITER, threads)
    tot_it, tot_t, kind, lat = 0, 0.0, "port", []
    for _ in range(args.steps):
        _, kind, n, dt, _ = cpu_reference_rate(p, y, NITER, threads)
        tot_it += n
        tot_t += dt
        lat.append(1000.0 * dt)
    value = tot_it / tot_t
    sample = (f"one full reconstruction ({NITER} PCG iterations) of the workload per step, {threads} host threads "
              f"over the independent (coil, segment) Gnufft calls")
    lat.sort()
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * tot_t / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": _config(), "impl": "reference",
            "impl_note": REFERENCE_IMPL if kind == "reference" else "oracle port of the reference CPU path",
            "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def image_parity(p, y_host, x_gpu, x_ref, threads: int):
    """Error of the timed reconstruction (the last timed step's image) against
    the reference CPU path's image of the same data, an FP64 solve over the
    reference's float operator (FP64 vectors, inner products and steps) and
    the FP64 oracle."""
    import oracle as O

    def rel_l2(a, b):
        a, b = np.asarray(a, np.complex128), np.asarray(b, np.complex128)
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    O.set_threads(threads)
    o32 = O.build_problem_op(p, 0)
    xw, _ = o32.pcg_fp64_solver(y_host, "quad", p.nx, p.ny, p.nz, p.beta, niter=NITER)
    o64 = O.build_problem_op(p, 1)
    x64, _ = o64.pcg(np.asarray(y_host, np.complex128), "quad", p.nx, p.ny, p.nz, p.beta, niter=NITER)
    O.set_threads(1)
    return {"rel_l2_vs_reference": rel_l2(x_gpu, x_ref), "rel_l2_vs_fp64": rel_l2(x_gpu, x64),
            "rel_l2_vs_fp64_solve_over_float_operator": rel_l2(x_gpu, xw),
            "reference_vs_fp64": rel_l2(x_ref, x64),
            "reference_vs_fp64_solve_over_float_operator": rel_l2(x_ref, xw),
            "note": "image after the workload's 20 iterations; CG on this problem amplifies operator rounding "
                    "(~1e-6) into ~1e-1 image differences by iteration 10-20, so every solve whose float "
                    "operator rounds differently, the reference's own FP64 counterpart included, lands this far "
                    "apart; the 3-iteration images agree within 1e-4 (tests)"}


# --------------------------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------------------------
def run_gpu_arm(args):
    from powergrid_b200.replicas import job_rate, max_over_ranks
    import ctypes as C

    import torch

    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    import powergrid_b200 as pg
    from powergrid_b200 import _lib
    from powergrid_b200._lib import P, Penalty, check

    from powergrid_b200 import build as B
    B.build()
    pg.init(local)
    L = _lib.load()
    p = _problem()
    M, n = p.kx.size, p.nimg
    G = pg.Gnufft(M, 2.0, p.nx, p.ny, 1, p.kx, p.ky, p.kz)
    A = pg.TimeSegmentation(G, p.fm, p.t, M, n, p.L, 1, 1)
    Sg = pg.SENSE(A, p.smap, M, n, p.nc)
    R = pg.QuadPenalty(p.nx, p.ny, 1, p.beta)

    stream = torch.cuda.Stream(device=dev)
    sp = P(stream.cuda_stream)
    xt = torch.from_numpy(p.x_true).to(dev)
    y = torch.empty(Sg.n_data, dtype=torch.complex64, device=dev)
    x = torch.empty(n, dtype=torch.complex64, device=dev)
    iters = torch.zeros(1, dtype=torch.int32, device=dev)
    with torch.cuda.stream(stream):
        Sg.forward(xt, out=y, stream=stream)
    stream.synchronize()
    pen = R._struct()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def solve():
        check(L.pg_pcg_solve_device(Sg.handle, None, None, P(y.data_ptr()), C.byref(pen), NITER, P(x.data_ptr()),
                                    P(iters.data_ptr()), sp))

    # Each timed step carries one CUDA event pair, around the adjoint gridding
    # (the roofline stage) of its last PCG iteration; the other stage times
    # come from extra profiled steps after the timed region.
    check(L.pg_profile_enable(1))
    check(L.pg_profile_only(b"adjoint_gridding"))
    sampler = ClockSampler(local)
    sampler.__enter__()
    for _ in range(max(3, args.warmup)):
        with torch.cuda.stream(stream):
            flush.zero_()
            solve()
    stream.synchronize()
    sampler.rows.clear()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    step_ms, spread_ms = [], []
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = _lib.launches()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[i][0].record(stream)
            solve()
            ev[i][1].record(stream)
        stream.synchronize()
        step_ms.append(ev[i][0].elapsed_time(ev[i][1]))
        ms = C.c_float()
        if L.pg_profile_stage_ms(b"adjoint_gridding", C.byref(ms)) == 0:
            spread_ms.append(ms.value)
    torch.cuda.synchronize()
    launches = _lib.launches() - launches0
    sampler.__exit__(None, None, None)

    stages = ["pre", "fft_fwd", "gather", "adjoint_gridding", "prep", "spread", "fft_adj", "post"]
    stage_ms = {k: [] for k in stages}
    check(L.pg_profile_only(None))
    for i in range(4):
        with torch.cuda.stream(stream):
            flush.zero_()
            solve()
        stream.synchronize()
        if i == 0:
            continue                      # the first profiled solve re-captures the graph
        for k in stages:
            ms = C.c_float()
            if L.pg_profile_stage_ms(k.encode(), C.byref(ms)) == 0:
                stage_ms[k].append(ms.value)
    check(L.pg_profile_enable(0))
    total_ms = sum(step_ms)
    done = int(iters.item())
    total_ms = max_over_ranks(total_ms, device=dev)
    value = job_rate(args.steps * NITER, total_ms / 1000.0, ws)

    # end to end through the C ABI host entry point (pinned host buffers)
    yh = torch.empty(Sg.n_data, dtype=torch.complex64).pin_memory()
    yh.copy_(y.cpu())
    xh = torch.empty(n, dtype=torch.complex64).pin_memory()
    itn = C.c_uint64()
    check(L.pg_pcg_solve(Sg.handle, None, None, P(yh.data_ptr()), C.byref(pen), NITER, P(xh.data_ptr()),
                         C.byref(itn)))
    e2e_steps = max(3, min(args.steps, 10))
    if ws > 1:
        torch.distributed.barrier()
    e2e_s = 0.0
    for _ in range(e2e_steps):
        flush.zero_()                      # L2 flushed before every step, as in the device-resident loop
        torch.cuda.synchronize()
        t0 = time.perf_counter()           # pg_pcg_solve returns after its D2H copy has landed
        check(L.pg_pcg_solve(Sg.handle, None, None, P(yh.data_ptr()), C.byref(pen), NITER, P(xh.data_ptr()),
                             C.byref(itn)))
        e2e_s += time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, device=dev)
    e2e = job_rate(e2e_steps * NITER, e2e_s, ws)

    # roofline of the adjoint gridding (clearing + spread): algorithmic bytes
    # per application = coils * (M * (4*d + 8 + 4) + L * G * 8), d = 2, G = 256^2
    G2 = (2 * p.nx) * (2 * p.ny)
    alg_bytes = p.nc * (M * (4 * 2 + 8 + 4) + p.L * G2 * 8)
    peak, peak_kind = _peaks()
    avg_spread = statistics.mean(spread_ms) if spread_ms else float("nan")
    achieved = alg_bytes / (avg_spread / 1000.0) / 1e9 if spread_ms else None
    traffic = None
    tp = os.path.join(ROOT, "profiles", "spread_cfg2_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get("bytes_per_launch")
        except Exception:
            traffic = None

    if rank == 0:
        cpu, parity = None, None
        if ws == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            y_host = y.cpu().numpy()
            rate, kind, nit, dt, x_ref = cpu_reference_rate(p, y_host, NITER, threads)
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
                   "sample": f"one full reconstruction ({nit} PCG iterations, {dt:.1f} s) of the same workload, "
                             f"{threads} host threads over independent (coil, segment) Gnufft calls"}
            parity = image_parity(p, y_host, x.cpu().numpy(), x_ref, threads)
        clocks = sampler.summary()
        lat = sorted(step_ms)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": _config(), "iterations_completed_last_step": done,
                "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
                "clocks": clocks,
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(Sg.n_data * 8),
                        "d2h_bytes_per_step": int(n * 8), "l2": "flushed before each step, outside the timed call",
                        "timer": "host clock around the synchronous pg_pcg_solve call (copies included)"},
                "stages_ms_per_launch": {k: (statistics.mean(v) if v else None) for k, v in stage_ms.items()},
                "roofline": {"kernel": "adjoint gridding: grid clearing + k_spread2d (TS-fused, 4 coils x 8 "
                                       "segments), one event pair around both",
                             "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                             "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_spread,
                             "peak_source": peak_kind},
                "cpu_baseline": cpu,
                "parity": parity,
                "gpu_launches": int(launches)}
        if ws == 1 and not args.no_serving:
            line["serving"] = run_serving()
        if ws == 1 and not args.no_gdft:
            line["gdft"] = gdft_block(5, 3, stream, with_error=not args.no_cpu_baseline)
        if ws == 1 and not args.no_secondary:
            # the other configurations' solve rates, measured in the same run: cfg1 (10-iteration 2-D
            # solves, launch-bound) and cfg5 (one 30-iteration 3-D pcSenseTimeSeg TV solve, ~20 s)
            line["secondary"] = {"cfg1": run_workload("cfg1", 20, 5), "cfg5": run_workload("cfg5", 1, 3)}
        print(json.dumps(line))
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_serving(n_requests: int = 16, rate_hz: float = 20.0, inflight: int = 8, seed: int = 4, small: bool = False):
    """Config 4: a seeded Poisson stream of time-segmented SENSE reconstructions of
    uneven size.  Three forms over the same stream:

      plain_one_at_a_time  the operator API used as the reference driver does
                           (PowerGridIsmrmrd.cpp:191-264): requests in arrival
                           order, and per slice Gnufft + TimeSegmentation + SENSE
                           construction and reconSolve (host buffers in and out);
      served               the request server with `inflight` slots (per-request
                           shared trajectory tables, jobs overlapping on streams);
      served_one_slot      the same server with one slot.
    Returns a summary dict."""
    import numpy as np

    import powergrid_b200 as pg
    from powergrid_b200 import synthetic as S
    from powergrid_b200.serve import ReconRequest, Server

    items = S.serving_stream(seed=seed, n_requests=n_requests, rate_hz=rate_hz, small=small)
    reqs = []
    for it in items:
        M, n = it.kx.size, it.nimg
        G = pg.Gnufft(M, 2.0, it.nx, it.ny, it.nz, it.kx, it.ky, it.kz)
        A = pg.TimeSegmentation(G, it.fm, it.t, M, n, it.L, 1, 1)
        Sg = pg.SENSE(A, it.smap, M, n, it.nc)
        y = Sg * it.x_true
        # unit-RMS data: the reference solver's |denom| guard (1e25) is scale
        # dependent and the unnormalised operators would trip it on big requests
        y = (y / np.sqrt(np.mean(np.abs(y) ** 2))).astype(np.complex64)
        del Sg, A, G
        reqs.append(ReconRequest(it.nx, it.ny, it.nz, it.nc, it.L, it.niter, it.beta, it.kx, it.ky, it.kz, it.t,
                                 np.tile(it.fm, it.n_slices), np.tile(it.smap, it.n_slices),
                                 np.tile(y, it.n_slices), it.n_slices))
    budget = 120 << 30

    def serve(slots):
        srv = Server(hbm_budget_bytes=budget, max_inflight=slots)
        t0 = time.perf_counter()
        tickets = []
        for it, r in zip(items, reqs):
            delay = it.arrival_s - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets.append(srv.submit(r))
        lat, iters, done, setup, solve = [], 0, 0.0, 0.0, 0.0
        for t in tickets:
            _, st = srv.wait(t)
            assert st["status"] == "PG_OK", st
            lat.append(st["t_done_ms"] - st["t_submit_ms"])
            iters += st["iters_done"]
            done = max(done, st["t_done_ms"])
            setup += st["setup_ms"]
            solve += st["solve_ms"]
        makespan = time.perf_counter() - t0
        srv.close()
        lat.sort()
        jobs = sum(r.n_slices for r in reqs)
        return {"iters_per_s": iters / makespan, "makespan_s": makespan, "iterations": iters,
                "latency_ms_p50": lat[len(lat) // 2], "latency_ms_p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                "mean_job_setup_ms": setup / jobs, "mean_job_solve_ms": solve / jobs}

    def direct():
        t0 = time.perf_counter()
        lat, iters = [], 0
        for it, r in zip(items, reqs):
            delay = it.arrival_s - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            M, n = it.kx.size, it.nimg
            R = pg.QuadPenalty(it.nx, it.ny, it.nz, it.beta)
            for sl in range(it.n_slices):
                G = pg.Gnufft(M, 2.0, it.nx, it.ny, it.nz, it.kx, it.ky, it.kz)
                A = pg.TimeSegmentation(G, r.field_map[sl * n:(sl + 1) * n], it.t, M, n, it.L, 1, 1)
                Sg = pg.SENSE(A, r.sense_map[sl * n * it.nc:(sl + 1) * n * it.nc], M, n, it.nc)
                _, k = pg.solve_pwls_pcg(None, Sg, None, r.data[sl * M * it.nc:(sl + 1) * M * it.nc], R, it.niter)
                iters += k
                Sg.close(); A.close(); G.close()
            lat.append(1000.0 * (time.perf_counter() - t0 - it.arrival_s))
        makespan = time.perf_counter() - t0
        lat.sort()
        return {"iters_per_s": iters / makespan, "makespan_s": makespan, "iterations": iters,
                "latency_ms_p50": lat[len(lat) // 2], "latency_ms_p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]}

    serve(inflight)  # warm-up: module loading, pool growth
    direct()         # warm-up: per-shape gridding tunings are cached for both forms
    plain = direct()
    served_one = serve(1)
    served = serve(inflight)
    dist = ("small requests: 32-48 in-plane, 1-2 slices, 2-4 coils, 2k-8k samples, L=3-4" if small else
            "64-256 in-plane (or 3-D 64-128 x 16-32), 1-32 slices, 4-32 coils, 8k-200k samples, L=4-12")
    return {"workload": f"config 4 stream: {n_requests} seeded requests, Poisson {rate_hz}/s, {dist}, "
                        f"{items[0].niter} PCG iterations, QuadPenalty, unit-RMS data; "
                        f"{sum(r.n_slices for r in reqs)} slice jobs",
            "plain_one_at_a_time": plain, "served_one_slot": served_one, "served": served, "inflight": inflight,
            "speedup_iters_per_s": served["iters_per_s"] / plain["iters_per_s"]}


SMS, SM_MAX_MHZ = 148, 1965.0


def gdft_block(steps: int, warmup: int, stream, with_error: bool = True):
    """Config 3: SENSE<Gdft> 64x64x32, 8 coils, 131072 samples; per step one
    forward and one adjoint on device buffers (CUDA events on the operator's
    stream).  Reports sample-voxel pairs/s per direction (all 8 coils share a
    pair's phase and sincos), the FP32 and MUFU rates those imply against the
    derived peaks (148 SMs x 128 FP32 lanes x 2 flops, 148 SMs x 16 MUFU ops,
    per clock at the 1965 MHz maximum), and, with_error, the error of 48
    sampled forward rows (coil 0) and 24 sampled adjoint voxels (8 coils)
    against the FP64 DFT."""
    import torch

    import powergrid_b200 as pg
    from powergrid_b200 import synthetic as S
    dev = torch.device("cuda", torch.cuda.current_device())
    p = S.config3()
    M, n = p.kx.size, p.nimg
    ix, iy, iz = S.image_coords(p.nx, p.ny, p.nz)
    G = pg.Gdft(M, n, p.kx, p.ky, p.kz, ix, iy, iz, p.fm, p.t)
    Sg = pg.SENSE(G, p.smap, M, n, p.nc)
    x = torch.from_numpy(p.x_true).to(dev)
    y = torch.empty(Sg.n_data, dtype=torch.complex64, device=dev)
    xa = torch.empty(n, dtype=torch.complex64, device=dev)
    torch.cuda.synchronize()
    for _ in range(warmup):
        Sg.forward(x, out=y, stream=stream)
        Sg.adjoint(y, out=xa, stream=stream)
    stream.synchronize()
    fwd, adj = [], []
    for _ in range(steps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        Sg.forward(x, out=y, stream=stream)
        e[1].record(stream)
        Sg.adjoint(y, out=xa, stream=stream)
        e[2].record(stream)
        stream.synchronize()
        fwd.append(e[0].elapsed_time(e[1]))
        adj.append(e[1].elapsed_time(e[2]))
    pairs = float(M) * n
    tf, ta = statistics.mean(fwd), statistics.mean(adj)
    clk = SM_MAX_MHZ * 1e6
    fp32_peak = SMS * 128 * 2 * clk
    mufu_peak = SMS * 16 * clk
    flops_pair = 8 * p.nc               # one complex multiply-add per coil
    res = {"workload": "cfg3 SENSE<Gdft> 64x64x32, 8 coils, 131072 samples, +-150 Hz, 0-25 ms readout",
           "metric": "sample-voxel pairs/s per direction (8 coils per pair)", "steps": steps, "warmup": warmup,
           "forward_ms": tf, "adjoint_ms": ta, "forward_pairs_per_s": pairs / (tf / 1e3),
           "adjoint_pairs_per_s": pairs / (ta / 1e3),
           "fp32_frac_of_derived_peak": {"forward": pairs * flops_pair / (tf / 1e3) / fp32_peak,
                                         "adjoint": pairs * flops_pair / (ta / 1e3) / fp32_peak},
           "mufu_frac_of_derived_peak": {"forward": pairs * 2 / (tf / 1e3) / mufu_peak,
                                         "adjoint": pairs * 2 / (ta / 1e3) / mufu_peak},
           "peaks": f"derived at {SM_MAX_MHZ:.0f} MHz: FP32 {fp32_peak / 1e12:.1f} TFLOP/s, MUFU "
                    f"{mufu_peak / 1e12:.2f} Tops/s (2 MUFU ops, sin and cos, and {flops_pair} FP32 flops per pair)"}
    if with_error:
        import oracle as O
        yh, xh = y.cpu().numpy(), xa.cpu().numpy()
        rng = np.random.default_rng(0)
        rows = np.sort(rng.choice(M, 48, replace=False))
        vox = np.sort(rng.choice(n, 24, replace=False))
        sm = p.smap.reshape(p.nc, n)
        f64 = O.gdft(2, p.kx[rows], p.ky[rows], p.kz[rows], ix, iy, iz, p.fm, p.t[rows])
        ref_f = f64.forward((sm[0] * p.x_true).astype(np.complex128))
        a64 = O.gdft(2, p.kx, p.ky, p.kz, ix[vox], iy[vox], iz[vox], p.fm[vox], p.t)
        ref_a = np.zeros(vox.size, np.complex128)
        for c in range(p.nc):
            ref_a += np.conj(sm[c, vox]).astype(np.complex128) * a64.adjoint(yh[c * M:(c + 1) * M].astype(np.complex128))

        def rel(a, b):
            return float(np.linalg.norm(np.asarray(a, np.complex128) - b) / np.linalg.norm(b))

        res["rel_l2_vs_fp64"] = {"forward_48_rows_coil0": rel(yh[rows], ref_f), "adjoint_24_voxels": rel(xh[vox], ref_a)}
    return res


def cpu_table():
    """The reference CPU path per configuration on this host: 1 thread and all
    host threads (independent units on threads; ctypes releases the GIL).
    Bounded samples, each stated: cfg1 a full 10-iteration solve; cfg2 a
    3-iteration solve on 1 thread (the solve's start, one forward, included)
    and a full 20-iteration solve on all threads; cfg3 the reference's float
    ftCpu / iftCpu on 64 sample rows (forward) or 64 voxels (adjoint) of all 8
    coils, as pairs/s; cfg5 one shot-coil-segment unit of the 3-D Gnufft
    (forward + adjoint, 131072 samples, 256x256x128 grid) scaled to a PCG
    iteration of 16 shots x 32 coils x 12 segments (two operator
    applications)."""
    import concurrent.futures as cf

    import oracle as O
    from powergrid_b200 import synthetic as S
    nth = os.cpu_count() or 1
    ref = O.reference_available()
    if ref:
        O.use_reference(True)
    out = {"host_threads": nth, "kind": "reference" if ref else "port"}

    def timed(fn):
        t0 = time.perf_counter()
        fn()
        return time.perf_counter() - t0

    p = S.config1()
    o = O.build_problem_op(p, 0)
    y = o.forward(p.x_true)
    O.set_threads(1)
    t1 = timed(lambda: o.pcg(y, "quad", p.nx, p.ny, 1, p.beta, niter=10))
    out["cfg1"] = {"metric": "PCG iters/s (10 iterations)", "cpu_1thr": 10 / t1,
                   "cpu_all": 10 / t1, "note": "one coil, no segments: no independent units to spread"}
    p = S.config2()
    o = O.build_problem_op(p, 0)
    O.set_threads(nth)
    y = o.forward(p.x_true)
    O.set_threads(1)
    t1 = timed(lambda: o.pcg(y, "quad", p.nx, p.ny, 1, p.beta, niter=3))
    O.set_threads(nth)
    ta = timed(lambda: o.pcg(y, "quad", p.nx, p.ny, 1, p.beta, niter=20))
    out["cfg2"] = {"metric": "PCG iters/s", "cpu_1thr": 3 / t1, "cpu_all": 20 / ta,
                   "sample": "1 thread: a 3-iteration solve; all threads: a 20-iteration solve"}
    O.set_threads(1)
    p = S.config3()
    M, n = p.kx.size, p.nimg
    ix, iy, iz = S.image_coords(p.nx, p.ny, p.nz)
    sm = p.smap.reshape(p.nc, n)
    rows = np.arange(0, M, M // 64)[:64]
    vox = np.arange(0, n, n // 64)[:64]
    fwd = O.gdft(0, p.kx[rows], p.ky[rows], p.kz[rows], ix, iy, iz, p.fm, p.t[rows])
    adj = O.gdft(0, p.kx, p.ky, p.kz, ix[vox], iy[vox], iz[vox], p.fm[vox], p.t)
    xs = [(sm[c] * p.x_true).astype(np.complex64) for c in range(p.nc)]
    yv = S.image(S.Rng(7), M)

    def fwd_all(pool):
        list(pool.map(lambda c: fwd.forward(xs[c]), range(p.nc)))

    def adj_all(pool):
        list(pool.map(lambda c: adj.adjoint(yv), range(p.nc)))

    g = {}
    for label, workers in (("cpu_1thr", 1), ("cpu_all", nth)):
        with cf.ThreadPoolExecutor(max_workers=workers) as pool:
            tf = timed(lambda: fwd_all(pool))
            ta = timed(lambda: adj_all(pool))
        g[label] = {"forward_pairs_per_s": rows.size * n / tf, "adjoint_pairs_per_s": vox.size * M / ta}
    out["cfg3"] = {"metric": "sample-voxel pairs/s per direction (8 coils per pair)", **g,
                   "sample": "64 sample rows (forward) / 64 voxels (adjoint), all 8 coils; all threads: coils "
                             "on threads (8 units)"}
    p = S.config5(shots=16, nc=1, per=2048)
    Mshot = p.kx.size // 16
    unit = O.gnufft(0, Mshot, p.nx, p.ny, p.nz, p.kx[:Mshot], p.ky[:Mshot], p.kz[:Mshot])
    xv = S.image(S.Rng(8), p.nimg)
    yv = unit.forward(xv)
    tu = timed(lambda: (unit.forward(xv), unit.adjoint(yv)))
    units = 16 * 32 * 12
    with cf.ThreadPoolExecutor(max_workers=nth) as pool:
        tpar = timed(lambda: list(pool.map(lambda k: (unit.forward(xv), unit.adjoint(yv)), range(nth))))
    out["cfg5"] = {"metric": "PCG iters/s (extrapolated)", "cpu_1thr": 1.0 / (units * tu),
                   "cpu_all": 1.0 / (units * tpar / nth),
                   "sample": f"one shot-coil-segment 3-D Gnufft forward+adjoint ({Mshot} samples, "
                             f"{2 * p.nx}x{2 * p.ny}x{2 * p.nz} grid) "
                             f"= {tu:.2f} s on 1 thread, {nth} such units concurrently in {tpar:.2f} s; x {units} "
                             "units per iteration"}
    if ref:
        O.use_reference(False)
    return out


def run_workload(name: str, steps: int, warmup: int):
    """Secondary workloads, one JSON line each (parity cases elsewhere, measured here).

    cfg3: SENSE<Gdft> 64x64x32, 8 coils, 131072 samples; per step one forward and
          one adjoint; reports sample-voxel pairs/s per direction.
    cfg5: pcSenseTimeSeg 128x128x64, 16 shots x 131072 samples, 32 coils, L=12,
          TVPenalty; PCG iterations/s over one solve of `niter` iterations.
    direct: spatial interpolation at gridos 3, density compensation and coil
          images on the cfg2 and cfg3 trajectories.
    """
    import ctypes as C

    import torch

    import powergrid_b200 as pg
    from powergrid_b200 import _lib
    from powergrid_b200 import synthetic as S
    from powergrid_b200._lib import check

    pg.init(0)
    dev = torch.device("cuda", 0)
    L = _lib.load()
    stream = torch.cuda.Stream(device=dev)
    sampler = ClockSampler(0)
    if name == "cfg1":
        p = S.config1()
        M, n = p.kx.size, p.nimg
        G = pg.Gnufft(M, 2.0, p.nx, p.ny, 1, p.kx, p.ky, p.kz)
        Sg = pg.SENSE(G, p.smap, M, n, 1)
        R = pg.QuadPenalty(p.nx, p.ny, 1, p.beta)
        x = torch.from_numpy(p.x_true).to(dev)
        y = torch.empty(Sg.n_data, dtype=torch.complex64, device=dev)
        Sg.forward(x, out=y, stream=stream)
        xo = torch.empty(n, dtype=torch.complex64, device=dev)
        it = torch.zeros(1, dtype=torch.int32, device=dev)
        for _ in range(warmup):
            pg.solve_pwls_pcg_device(Sg, y, R, p.niter, xo, iters=it, stream=stream)
        stream.synchronize()
        ms = []
        with sampler:
            for _ in range(steps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                pg.solve_pwls_pcg_device(Sg, y, R, p.niter, xo, iters=it, stream=stream)
                e1.record(stream)
                stream.synchronize()
                ms.append(e0.elapsed_time(e1))
        return {"workload": "cfg1 SENSE<Gnufft> 64x64, 1 coil, 4096 samples, QuadPenalty 1e-3, 10 PCG iterations",
                "metric": METRIC, "unit": UNIT, "value": p.niter / (statistics.mean(ms) / 1e3),
                "ms_per_solve": statistics.mean(ms), "steps": steps, "warmup": warmup, "clocks": sampler.summary()}
    if name == "cfg3":
        with sampler:
            res = gdft_block(steps, warmup, stream, with_error=True)
        res["clocks"] = sampler.summary()
        return res
    if name == "cfg5":
        p = S.config5()
        op = pg.pcSenseTimeSeg(p.kx, p.ky, p.kz, p.nx, p.ny, p.nz, p.nc, p.t, p.L, 1, p.smap, p.fm, p.pmap)
        R = pg.TVPenalty(p.nx, p.ny, p.nz, p.beta, p.delta)
        x = torch.from_numpy(p.x_true).to(dev)
        y = torch.empty(op.n_data, dtype=torch.complex64, device=dev)
        torch.cuda.synchronize()
        op.forward(x, out=y, stream=stream)
        stream.synchronize()
        # The solver's |denominator| guard (1e25) is scale dependent and the
        # unnormalised 3-D operator is large: scale the data so that the first
        # line-search denominator ||A A' y||^2 is 1.
        g = torch.empty(p.nimg, dtype=torch.complex64, device=dev)
        op.adjoint(y, out=g, stream=stream)
        Ag = torch.empty_like(y)
        op.forward(g, out=Ag, stream=stream)
        stream.synchronize()
        y /= float(torch.sqrt(torch.sum(torch.abs(Ag).double() ** 2)))
        del g, Ag
        xo = torch.empty(p.nimg, dtype=torch.complex64, device=dev)
        it = torch.zeros(1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        for _ in range(warmup):
            pg.solve_pwls_pcg_device(op, y, R, 2, xo, iters=it, stream=stream)
        stream.synchronize()
        ms, done = [], 0
        check(L.pg_profile_enable(1))
        with sampler:
            for _ in range(steps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                pg.solve_pwls_pcg_device(op, y, R, p.niter, xo, iters=it, stream=stream)
                e1.record(stream)
                stream.synchronize()
                ms.append(e0.elapsed_time(e1))
                done += int(it.item())
        stages = {}
        for k in ["pre", "fft_fwd", "gather", "prep", "spread", "fft_adj", "post"]:
            v = C.c_float()
            if L.pg_profile_stage_ms(k.encode(), C.byref(v)) == 0:
                stages[k] = v.value
        check(L.pg_profile_enable(0))
        return {"workload": "cfg5 pcSenseTimeSeg 128x128x64, 16 shots x 131072 samples, 32 coils, L=12, "
                            f"TVPenalty (beta {p.beta}, delta {p.delta}), data scaled so that the first "
                            f"line-search denominator is 1, {p.niter} PCG iterations",
                "metric": METRIC, "unit": UNIT, "value": done / (sum(ms) / 1e3), "iterations": done,
                "ms_per_solve": statistics.mean(ms), "steps": steps, "warmup": warmup,
                "stage_ms_last_launch": stages, "clocks": sampler.summary()}
    if name == "direct":
        res = {"workload": "direct reconstruction pieces on the cfg2 (128x128, 131072 samples) and cfg3 "
                           "(64x64x32, 131072 samples) trajectories: spatial interpolation on the 3x oversampled "
                           "grid (device buffers, CUDA events), density compensation and 4-coil gridded images "
                           "through the host-buffer API (wall clock, set-up included)",
               "steps": steps, "warmup": warmup}
        with sampler:
            for tag, p in (("2d", S.config2()), ("3d", S.config3())):
                M = p.kx.size
                G3 = pg.Gnufft(M, 3.0, p.nx, p.ny, p.nz, p.kx, p.ky, p.kz)
                ng = G3.grid_length
                d = torch.ones(M, dtype=torch.complex64, device=dev)
                grid = torch.empty(ng, dtype=torch.complex64, device=dev)
                yv = torch.empty(M, dtype=torch.complex64, device=dev)
                sp = C.c_void_p(stream.cuda_stream)
                args_a = (G3.handle, C.c_void_p(d.data_ptr()), C.c_void_p(grid.data_ptr()), sp)
                args_f = (G3.handle, C.c_void_p(grid.data_ptr()), C.c_void_p(yv.data_ptr()), sp)
                torch.cuda.synchronize()
                for _ in range(warmup):
                    check(L.pg_gnufft_adjoint_spatial_interp_device(*args_a))
                    check(L.pg_gnufft_forward_spatial_interp_device(*args_f))
                stream.synchronize()
                ta, tf = [], []
                for _ in range(steps):
                    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                    e[0].record(stream)
                    check(L.pg_gnufft_adjoint_spatial_interp_device(*args_a))
                    e[1].record(stream)
                    check(L.pg_gnufft_forward_spatial_interp_device(*args_f))
                    e[2].record(stream)
                    stream.synchronize()
                    ta.append(e[0].elapsed_time(e[1]))
                    tf.append(e[1].elapsed_time(e[2]))
                del G3
                t0 = time.perf_counter()
                dcf = pg.calc3DDensityCompensation(p.kx, p.ky, p.kz, p.nx, p.nz)
                t_dcf = time.perf_counter() - t0
                G2 = pg.Gnufft(M, 2.0, p.nx, p.ny, p.nz, p.kx, p.ky, p.kz)
                data = S.image(S.Rng(9), M * 4)
                pg.gridCoilImages(G2, dcf, data, 4)  # warm (plans, workspaces)
                t0 = time.perf_counter()
                imgs = pg.gridCoilImages(G2, dcf, data, 4)
                t_img = time.perf_counter() - t0
                pg.calcSumOfSquaresImage(imgs, 4)
                del G2
                dim = 3 if p.nz > 1 else 2
                a_ms, f_ms = statistics.mean(ta), statistics.mean(tf)
                res[tag] = {"samples": M, "grid_cells_os3": ng,
                            "adjoint_interp_ms": a_ms, "forward_interp_ms": f_ms,
                            "adjoint_interp_samples_per_s": M / (a_ms / 1e3),
                            "adjoint_interp_algorithmic_GBps": (M * (4 * dim + 8) + ng * 8) / (a_ms / 1e3) / 1e9,
                            "density_compensation_host_call_s": t_dcf,
                            "coil_images_4_host_call_s": t_img}
        res["clocks"] = sampler.summary()
        return res
    raise SystemExit(f"unknown workload {name}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the config-4 serving stream")
    ap.add_argument("--no-gdft", action="store_true", help="skip the config-3 Gdft block")
    ap.add_argument("--no-secondary", action="store_true", help="skip the cfg1 and cfg5 solve-rate blocks")
    ap.add_argument("--serving-only", action="store_true", help="only the config-4 serving stream")
    ap.add_argument("--workload", default=None, choices=["cfg1", "cfg3", "cfg5", "direct", "cpu"],
                    help="a secondary workload instead")
    args = ap.parse_args()
    if args.workload == "cpu":
        print(json.dumps(cpu_table()))
        return 0
    if args.workload:
        print(json.dumps(run_workload(args.workload, args.steps, max(3, args.warmup))))
        return 0
    if args.serving_only:
        import powergrid_b200 as pg
        pg.init(0)
        print(json.dumps({"serving": run_serving(),
                          "serving_small": run_serving(n_requests=64, rate_hz=10000.0, small=True)}))
        return 0
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
