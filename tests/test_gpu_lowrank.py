"""The low-rank (partial separability) model on the GPU: LRobj over per-image
pcSenseTimeSeg / pcSENSE plans, the R_lowRank penalty wrapper, and the PWLS-PCG
solve that composes them (lowRank/oscillateRecon.cpp:256-265), each against
the oracle's restatement of lowRank/LRobj.cpp and lowRank/R_lowRank.cpp over
the oracle's operators.

Tolerances (relative L2): operator application and penalty pieces <= 1e-5,
a 5-iteration solve <= 1e-4 with the same number of completed iterations.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

OP_TOL = 1e-5
PCG_TOL = 1e-4


def _basis(rank, nimg, seed):
    """vLR = trans(v.cols(0, rank-1)) of an orthonormal temporal basis v
    (oscillateRecon.cpp:160-161): rank x nimg."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((nimg, nimg)) + 1j * rng.standard_normal((nimg, nimg))
    q, _ = np.linalg.qr(a)
    return np.ascontiguousarray(q[:, :rank].conj().T).astype(np.complex64)


def _reps_timeseg(pg, oracle, n, nimg, ns=2, nc=2, L=3, per=512):
    """One pcSenseTimeSeg per repetition (its own interleaves and shot phases),
    on the device and in the oracle."""
    from powergrid_b200 import synthetic as S
    fm = S.field_map(S.Rng(201), n, n, 1, 60.0)
    sm = S.coil_maps(S.Rng(202), n, n, 1, nc)
    dev, ref = [], []
    for r in range(nimg):
        kxs, kys, ts = [], [], []
        for s in range(ns):
            a, b, t = S.spiral(n, ns * nimg, per, 8e-3, which=[r * ns + s])
            kxs.append(a); kys.append(b); ts.append(t)
        kx, ky, t = (np.concatenate(v) for v in (kxs, kys, ts))
        kz = np.zeros_like(kx)
        pm = S.shot_phase_maps(S.Rng(210 + r), n, n, 1, ns)
        dev.append(pg.pcSenseTimeSeg(kx, ky, kz, n, n, 1, nc, t, L, 1, sm, fm, pm))
        ref.append(oracle.pcsense_timeseg(0, kx, ky, kz, n, n, 1, nc, t, L, sm, fm, pm))
    return dev, ref


def _reps_gdft(pg, oracle, n, nz, nimg, ns=2, nc=2, per=96):
    from powergrid_b200 import synthetic as S
    fm = S.field_map(S.Rng(221), n, n, nz, 100.0)
    sm = S.coil_maps(S.Rng(222), n, n, nz, nc)
    dev, ref = [], []
    for r in range(nimg):
        kxs, kys, kzs, ts = [], [], [], []
        for s in range(ns):
            a, b, c, d = S.stack_of_spirals(n, nz, ns * nimg, per, 10e-3, which=[r * ns + s])
            kxs.append(a); kys.append(b); kzs.append(c); ts.append(d)
        kx, ky, kz, t = (np.concatenate(v) for v in (kxs, kys, kzs, ts))
        pm = S.shot_phase_maps(S.Rng(230 + r), n, n, nz, ns)
        dev.append(pg.pcSENSE(kx, ky, kz, n, n, nz, nc, t, sm, fm, pm))
        ref.append(oracle.pcsense(0, kx, ky, kz, n, n, nz, nc, t, sm, fm, pm))
    return dev, ref


def test_lrobj_over_pcsense_timeseg_vs_oracle(pg, oracle):
    """LRobj<pcSenseTimeSeg> 32x32, rank 2 of 3 repetitions, 2 shots x 2 coils, L=3."""
    from powergrid_b200 import synthetic as S
    n, nimg, rank = 32, 3, 2
    dev, ref = _reps_timeseg(pg, oracle, n, nimg)
    v = _basis(rank, nimg, 5)
    N, Nd = n * n, dev[0].n_data
    A = pg.LRobj(N, Nd, rank, nimg, v, dev)
    R = oracle.lowrank(N, Nd, rank, nimg, v, ref)
    assert (A.n_data, A.n_image) == (Nd * nimg, N * rank) == (R.n_data, R.n_image)
    x = np.concatenate([S.image(S.Rng(240 + k), N) for k in range(rank)])
    y = R.forward(x)
    ef, ea = rel_l2(A * x, y), rel_l2(A / y, R.adjoint(y))
    print(f"LRobj<pcSenseTimeSeg>: forward {ef:.2e}, adjoint {ea:.2e}")
    assert ef <= OP_TOL and ea <= OP_TOL


def test_lrobj_over_pcsense_vs_oracle(pg, oracle):
    """LRobj<pcSENSE> 16x16x2, rank 2 of 2 repetitions."""
    from powergrid_b200 import synthetic as S
    n, nz, nimg, rank = 16, 2, 2, 2
    dev, ref = _reps_gdft(pg, oracle, n, nz, nimg)
    v = _basis(rank, nimg, 6)
    N, Nd = n * n * nz, dev[0].n_data
    A = pg.LRobj(N, Nd, rank, nimg, v, dev)
    R = oracle.lowrank(N, Nd, rank, nimg, v, ref)
    x = np.concatenate([S.image(S.Rng(250 + k), N) for k in range(rank)])
    y = R.forward(x)
    ef, ea = rel_l2(A * x, y), rel_l2(A / y, R.adjoint(y))
    print(f"LRobj<pcSENSE>: forward {ef:.2e}, adjoint {ea:.2e}")
    assert ef <= OP_TOL and ea <= OP_TOL


@pytest.mark.parametrize("kind", ["quad", "tv"])
def test_r_lowrank_pieces_vs_oracle(pg, oracle, kind):
    """R_lowRank::Gradient (rank-fastest layout) and ::Denom (beta twice), 16x16x4, rank 3."""
    import torch
    from powergrid_b200 import synthetic as S
    nx = ny = 16
    nz, rank = 4, 3
    N = nx * ny * nz
    beta, delta = 0.3, 0.05
    v = _basis(rank, rank, 7)
    Rb = pg.QuadPenalty(nx, ny, nz, beta) if kind == "quad" else pg.TVPenalty(nx, ny, nz, beta, delta)
    Rl = pg.R_lowRank(Rb, rank, rank, v)
    x = np.concatenate([S.image(S.Rng(260 + k), N) for k in range(rank)])
    d = np.concatenate([S.image(S.Rng(270 + k), N) for k in range(rank)])
    xt, dt = torch.from_numpy(x).cuda(), torch.from_numpy(d).cuda()
    g = Rl.Gradient(xt).cpu().numpy()
    g_ref = oracle.lowrank_gradient(0, kind, nx, ny, nz, beta, delta, 3, rank, v, x)
    den = Rl.Denom(dt, xt)
    den_ref = oracle.lowrank_denom(0, kind, nx, ny, nz, beta, delta, 3, rank, v, d, x)
    eg = rel_l2(g, g_ref)
    ed = abs(den - den_ref.real) / abs(den_ref.real)
    print(f"R_lowRank {kind}: gradient {eg:.2e}, denom {ed:.2e}")
    assert eg <= OP_TOL and ed <= OP_TOL and abs(den_ref.imag) <= 1e-6 * abs(den_ref.real)


@pytest.mark.parametrize("kind", ["quad", "tv"])
def test_lowrank_pcg_vs_oracle(pg, oracle, kind):
    """solve_pwls_pcg<LRobj<pcSenseTimeSeg>, R_lowRank> 32x32, rank 3 of 3 repetitions,
    5 iterations, against the oracle's solve over the oracle's operators."""
    from powergrid_b200 import synthetic as S
    n, nimg = 32, 3
    rank = nimg
    dev, ref = _reps_timeseg(pg, oracle, n, nimg)
    v = _basis(rank, nimg, 8)
    N, Nd = n * n, dev[0].n_data
    A = pg.LRobj(N, Nd, rank, nimg, v, dev)
    Ao = oracle.lowrank(N, Nd, rank, nimg, v, ref)
    x_true = np.concatenate([S.image(S.Rng(280 + k), N) for k in range(rank)])
    y = Ao.forward(x_true)
    y = (y + 0.01 * np.abs(y).mean() * S.image(S.Rng(290), y.size)).astype(np.complex64)
    beta = 1e-2
    Rb = pg.QuadPenalty(n, n, 1, beta) if kind == "quad" else pg.TVPenalty(n, n, 1, beta, 0.1)
    x, it = pg.solve_pwls_pcg(None, A, None, y, pg.R_lowRank(Rb, rank, nimg, v), 5)
    xo, ito = oracle.pcg_lowrank(Ao, y, kind, n, n, 1, beta, rank, v, delta=0.1, niter=5)
    e = rel_l2(x, xo)
    print(f"low-rank PCG {kind}: {it} vs {ito} iterations, rel {e:.2e}")
    assert it == ito and e <= PCG_TOL


def test_lowrank_pcg_graph_reuse_and_eager(pg, oracle, monkeypatch):
    """The captured iteration stays cached on the LRobj: a second solve with
    another penalty basis rewrites the graph's basis matrices in place and must
    match the oracle's solve with that basis; the same solve with graphs off
    (the same kernels launched one by one, on a fresh LRobj) gives the same
    image up to the order of the gridding's float atomics."""
    from powergrid_b200 import synthetic as S
    n, nimg = 32, 3
    rank, beta, niter = nimg, 1e-2, 6
    dev, ref = _reps_timeseg(pg, oracle, n, nimg)
    v, v2 = _basis(rank, nimg, 8), _basis(rank, nimg, 11)
    N, Nd = n * n, dev[0].n_data
    A = pg.LRobj(N, Nd, rank, nimg, v, dev)
    Ao = oracle.lowrank(N, Nd, rank, nimg, v, ref)
    y = Ao.forward(np.concatenate([S.image(S.Rng(300 + k), N) for k in range(rank)])).astype(np.complex64)

    def pen(vb):
        return pg.R_lowRank(pg.TVPenalty(n, n, 1, beta, 0.1), rank, nimg, vb)

    for vb in (v, v2):
        x, it = pg.solve_pwls_pcg(None, A, None, y, pen(vb), niter)
        xo, ito = oracle.pcg_lowrank(Ao, y, "tv", n, n, 1, beta, rank, vb, delta=0.1, niter=niter)
        e = rel_l2(x, xo)
        print(f"cached low-rank PCG: {it} vs {ito} iterations, rel {e:.2e}")
        assert it == ito and e <= PCG_TOL
    monkeypatch.setenv("PG_NO_GRAPH", "1")
    A2 = pg.LRobj(N, Nd, rank, nimg, v, dev)
    x2, it2 = pg.solve_pwls_pcg(None, A2, None, y, pen(v2), niter)
    e2 = rel_l2(x2, x)
    print(f"eager vs graph: {e2:.2e}")
    assert it2 == it and e2 <= OP_TOL


def test_lowrank_invalid_inputs(pg, oracle):
    """The reference's R_lowRank gradient needs rank == images; LRobj needs one
    operator of the stated shape per image."""
    n, nimg = 32, 3
    dev, _ = _reps_timeseg(pg, oracle, n, nimg, per=256)
    N, Nd = n * n, dev[0].n_data
    v = _basis(2, nimg, 9)
    A = pg.LRobj(N, Nd, 2, nimg, v, dev)
    y = np.zeros(A.n_data, np.complex64)
    with pytest.raises(RuntimeError, match="rank == the number of images"):
        pg.solve_pwls_pcg(None, A, None, y, pg.R_lowRank(pg.QuadPenalty(n, n, 1, 1e-3), 2, nimg, v), 2)
    with pytest.raises(ValueError):
        pg.LRobj(N, Nd, 2, nimg, v, dev[:2])
    with pytest.raises(RuntimeError, match="the model needs"):
        pg.LRobj(N, Nd + 1, 2, nimg, v, dev)
    with pytest.raises(RuntimeError, match="does not match"):
        v3 = _basis(3, 3, 10)
        A3 = pg.LRobj(N, Nd, 3, 3, v3, dev)
        pg.solve_pwls_pcg(None, A3, None, np.zeros(A3.n_data, np.complex64),
                          pg.R_lowRank(pg.QuadPenalty(n, n, 2, 1e-3), 3, 3, v3), 2)
