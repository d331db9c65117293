"""Request server: continuous batching with HBM-footprint admission.

GPU tests check that a request's result is the same whether it runs alone
or overlapped with others (within the operator tolerance), that requests
exceeding the budget are rejected, and that cancellation ends a request.
The footprint model is host-only and tested on CPU.
"""
import numpy as np
import pytest

from conftest import rel_l2

MIX_TOL = 1e-5


def _requests(pg_mod, items):
    """Form each request's data with the GPU forward operator of its own geometry."""
    from powergrid_b200.serve import ReconRequest
    reqs = []
    for it in items:
        M, n = it.kx.size, it.nimg
        G = pg_mod.Gnufft(M, 2.0, it.nx, it.ny, it.nz, it.kx, it.ky, it.kz)
        A = pg_mod.TimeSegmentation(G, it.fm, it.t, M, n, it.L, 1, 1)
        S = pg_mod.SENSE(A, it.smap, M, n, it.nc)
        y = S * it.x_true
        reqs.append(ReconRequest(it.nx, it.ny, it.nz, it.nc, it.L, it.niter, it.beta, it.kx, it.ky, it.kz, it.t,
                                 np.tile(it.fm, it.n_slices), np.tile(it.smap, it.n_slices),
                                 np.tile(y, it.n_slices), it.n_slices))
    return reqs


def test_footprint_model_is_monotone():
    from powergrid_b200 import build as B
    B.build()
    from powergrid_b200.serve import ReconRequest, Server
    z = np.zeros(1, np.float32)

    def req(n, nc, M, L):
        k = np.zeros(M, np.float32)
        return ReconRequest(n, n, 1, nc, L, 10, 1e-3, k, k, k, k, np.zeros(n * n, np.float32),
                            np.zeros(n * n * nc, np.complex64), np.zeros(M * nc, np.complex64))

    base = Server.footprint(req(64, 4, 8192, 4))
    assert base > 0
    assert Server.footprint(req(128, 4, 8192, 4)) > base
    assert Server.footprint(req(64, 8, 8192, 4)) > base
    assert Server.footprint(req(64, 4, 65536, 4)) > base
    assert Server.footprint(req(64, 4, 8192, 8)) > base
    _ = z


@pytest.mark.gpu
def test_alone_equals_in_mix(pg):
    from powergrid_b200 import synthetic as S
    from powergrid_b200.serve import Server
    items = S.serving_stream(seed=11, n_requests=6, small=True, niter=5)
    reqs = _requests(pg, items)
    alone = []
    srv1 = Server(hbm_budget_bytes=8 << 30, max_inflight=1)
    for r in reqs:
        img, st = srv1.wait(srv1.submit(r))
        assert st["status"] == "PG_OK" and st["iters_done"] == 5 * r.n_slices
        alone.append(img.copy())
    srv1.close()
    srv = Server(hbm_budget_bytes=8 << 30, max_inflight=6)
    tickets = [srv.submit(r) for r in reqs]
    for r, t, a in zip(reqs, tickets, alone):
        img, st = srv.wait(t)
        assert st["status"] == "PG_OK"
        for s in range(r.n_slices):
            e = rel_l2(img[s], a[s])
            assert e <= MIX_TOL, e
    srv.close()


@pytest.mark.gpu
def test_results_match_direct_api(pg):
    """A served slice equals reconSolve through the operator API."""
    from powergrid_b200 import synthetic as S
    from powergrid_b200.serve import Server
    it = S.serving_stream(seed=12, n_requests=1, small=True, niter=5)[0]
    r = _requests(pg, [it])[0]
    srv = Server(hbm_budget_bytes=8 << 30, max_inflight=2)
    img, st = srv.wait(srv.submit(r))
    srv.close()
    M, n = it.kx.size, it.nimg
    G = pg.Gnufft(M, 2.0, it.nx, it.ny, it.nz, it.kx, it.ky, it.kz)
    A = pg.TimeSegmentation(G, it.fm, it.t, M, n, it.L, 1, 1)
    Sg = pg.SENSE(A, it.smap, M, n, it.nc)
    x = pg.reconSolve(r.data[: M * it.nc], Sg, pg.QuadPenalty(it.nx, it.ny, it.nz, it.beta), niter=5)
    assert rel_l2(img[0], x) <= MIX_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("n", [32, 40])
def test_batched_slices_match_per_slice_solves(pg, n):
    """The slices of a request are solved as one stacked operator with per-slice
    inner products and steps; each served slice equals the solve of that slice
    alone through the operator API (reconSolve over its own SENSE<TS<Gnufft>>),
    with slices that differ in field map, coil maps and data.  n = 32 runs the
    own FFT passes, n = 40 the cuFFT path; a budget just above one slice's
    footprint splits the request into one job per slice."""
    from powergrid_b200 import synthetic as S
    from powergrid_b200.serve import ReconRequest, Server
    ns, nc, L, niter, beta = 3, 3, 4, 6, 1e-3
    kx, ky, t = S.spiral(n, 4, 768, 10e-3)
    kz = np.zeros_like(kx)
    M, N = kx.size, n * n
    fms = [S.field_map(S.Rng(200 + k), n, n, 1, 100.0) for k in range(ns)]
    sms = [S.coil_maps(S.Rng(210 + k), n, n, 1, nc) for k in range(ns)]
    ops, ys = [], []
    for k in range(ns):
        G = pg.Gnufft(M, 2.0, n, n, 1, kx, ky, kz)
        A = pg.TimeSegmentation(G, fms[k], t, M, N, L, 1, 1)
        Sg = pg.SENSE(A, sms[k], M, N, nc)
        ops.append((G, A, Sg))
        ys.append((Sg * S.image(S.Rng(220 + k), N)).astype(np.complex64))
    r = ReconRequest(n, n, 1, nc, L, niter, beta, kx, ky, kz, t, np.concatenate(fms), np.concatenate(sms),
                     np.concatenate(ys), ns)
    direct = [pg.reconSolve(ys[k], ops[k][2], pg.QuadPenalty(n, n, 1, beta), niter=niter) for k in range(ns)]
    for budget, jobs in ((8 << 30, 1), (Server.footprint(r) + (64 << 10), ns)):
        srv = Server(hbm_budget_bytes=budget, max_inflight=2)
        img, st = srv.wait(srv.submit(r))
        srv.close()
        assert st["status"] == "PG_OK" and st["iters_done"] == ns * niter and st["jobs"] == jobs
        for k in range(ns):
            e = rel_l2(img[k], direct[k])
            print(f"n={n} budget {budget >> 20} MiB slice {k}: served vs alone {e:.2e}")
            assert e <= MIX_TOL


@pytest.mark.gpu
def test_admission_rejects_oversized_request(pg):
    from powergrid_b200 import synthetic as S
    from powergrid_b200._lib import PGError
    from powergrid_b200.serve import Server
    r = _requests(pg, S.serving_stream(seed=13, n_requests=1, small=True))[0]
    srv = Server(hbm_budget_bytes=Server.footprint(r) - 1, max_inflight=2)
    with pytest.raises(PGError, match="REJECTED"):
        srv.submit(r)
    srv.close()


@pytest.mark.gpu
def test_cancel_queued_request(pg):
    from powergrid_b200 import synthetic as S
    from powergrid_b200.serve import Server
    reqs = _requests(pg, S.serving_stream(seed=14, n_requests=3, small=True, niter=20))
    srv = Server(hbm_budget_bytes=8 << 30, max_inflight=1)
    t = [srv.submit(r) for r in reqs]
    srv.cancel(t[2])
    _, st2 = srv.wait(t[2])
    assert st2["status"] == "PG_CANCELLED"
    _, st0 = srv.wait(t[0])
    assert st0["status"] == "PG_OK"
    srv.close()


def _acquisition_dataset(pg_mod, n, nc, niter, beta, L):
    """A dataset of 2 slices x 2 contrasts x 2 repetitions, each image 4 spiral
    shots (one acquisition per shot), listed in a shuffled order.  Contrast 1
    uses a rotated trajectory, so the images form two trajectory groups.
    Returns the acquisitions, the limits, the maps, and per image (in the
    driver's loop order) its direct reconSolve through the operator API."""
    import math
    from powergrid_b200 import ingest as I
    from powergrid_b200 import synthetic as S
    shots, per = 4, 768
    N = n * n
    fms = np.stack([S.field_map(S.Rng(300 + s), n, n, 1, 80.0) for s in range(2)])
    sms = np.stack([S.coil_maps(S.Rng(310 + s), n, n, 1, nc) for s in range(2)])
    trajs = []
    for ec in range(2):
        kx, ky, t = S.spiral(n, shots, per, 10e-3)
        if ec == 1:
            c, s_ = math.cos(0.3), math.sin(0.3)
            kx, ky = (c * kx - s_ * ky).astype(np.float32), (s_ * kx + c * ky).astype(np.float32)
        trajs.append((kx, ky, np.zeros_like(kx), t))
    acqs, direct = [], []
    for sl in range(2):
        for ec in range(2):
            for rp in range(2):
                kx, ky, kz, t = trajs[ec]
                M = kx.size
                G = pg_mod.Gnufft(M, 2.0, n, n, 1, kx, ky, kz)
                Lk = L if L else int(math.ceil(float(np.float32(t.max() - t.min())) / 2e-3))
                A = pg_mod.TimeSegmentation(G, fms[sl], t, M, N, Lk, 1, 1)
                Sg = pg_mod.SENSE(A, sms[sl].ravel(), M, N, nc)
                y = (Sg * S.image(S.Rng(320 + 4 * sl + 2 * ec + rp), N)).astype(np.complex64)
                direct.append(((sl, ec, rp), pg_mod.reconSolve(y, Sg, pg_mod.QuadPenalty(n, n, 1, beta),
                                                                niter=niter)))
                yc = y.reshape(nc, shots, per)
                for sh in range(shots):
                    sel = slice(sh * per, (sh + 1) * per)
                    traj = np.stack([kx[sel], ky[sel], kz[sel], t[sel]], axis=1)
                    acqs.append(I.Acquisition(sh, 0, sl, rp, 0, ec, 0, yc[:, sh, :], traj))
    order = np.random.default_rng(5).permutation(len(acqs))
    limits = (shots, 1, 2, 2, 1, 2, 1)
    return [acqs[i] for i in order], limits, fms, sms, direct


@pytest.mark.gpu
@pytest.mark.parametrize("L", [0, 3])
def test_acquisition_request_matches_per_image_solves(pg, L):
    """pg_submit_acquisitions: every image of the index, gathered as
    getCompleteISMRMRDAcqData does, in the driver's loop order (slice,
    phase, contrast, average, repetition), equals the solve of that image
    alone; L = 0 takes the driver's default segment count."""
    from powergrid_b200 import ingest as I
    from powergrid_b200.serve import Server
    n, nc, niter, beta = 32, 3, 5, 1e-3
    from powergrid_b200.serve import ReconRequest
    acqs, limits, fms, sms, direct = _acquisition_dataset(pg, n, nc, niter, beta, L)
    track = I.acqTracking(acqs, limits)
    z = np.zeros(4 * 768, np.float32)
    one = ReconRequest(n, n, 1, nc, L or 5, niter, beta, z, z, z, z, fms[0], sms[0].ravel(),
                       np.zeros(z.size * nc, np.complex64))
    # two trajectory groups of 4 images: one job each, or one job per image
    for budget, jobs in ((8 << 30, 2), (Server.footprint(one) + (64 << 10), 8)):
        srv = Server(hbm_budget_bytes=budget, max_inflight=2)
        t = srv.submit_acquisitions(track, n, n, 1, fms, sms, L=L, niter=niter, beta=beta)
        img, st = srv.wait(t)
        srv.close()
        assert st["status"] == "PG_OK", st["error"]
        assert img.shape == (8, n * n) and st["iters_done"] == 8 * niter and st["jobs"] == jobs
        # loop order: slice, phase (1), contrast, average (1), repetition
        for k, ((sl, ec, rp), x) in enumerate(direct):
            assert k == (sl * 2 + ec) * 2 + rp
            e = rel_l2(img[k], x)
            print(f"L={L} budget {budget >> 20} MiB image {k}: served vs alone {e:.2e}")
            assert e <= MIX_TOL


@pytest.mark.gpu
def test_acquisition_request_rejects_missing_image(pg):
    from powergrid_b200 import ingest as I
    from powergrid_b200._lib import PGError
    from powergrid_b200.serve import Server
    n, nc = 32, 3
    acqs, limits, fms, sms, _ = _acquisition_dataset(pg, n, nc, 1, 1e-3, 3)
    # drop every acquisition of slice 1, contrast 0, repetition 1
    kept = [a for a in acqs if not (a.slice == 1 and a.contrast == 0 and a.repetition == 1)]
    track = I.acqTracking(kept, limits)
    srv = Server(hbm_budget_bytes=8 << 30, max_inflight=1)
    with pytest.raises(PGError, match="no acquisitions"):
        srv.submit_acquisitions(track, n, n, 1, fms, sms, L=3, niter=1, beta=1e-3)
    srv.close()
