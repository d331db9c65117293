"""The oversampled-FFT stage in both of its forms, and gridding edge cases.

Operators on power-of-two 2N grids (2-D and 3-D) run the library's own
pruned FFT passes (with the pre/post kernels fused in); PG_CUFFT=1 at
construction keeps the cuFFT form.  Both must agree with each other and with
the reference CPU path at the supported grid sizes (in-plane 64 ... 1024, z
16 ... 128 here), and the gridding must handle the
trajectory edges the reference's clamped windows define (samples on the
-N/2 border, a single sample, all samples in one tile).

Tolerances (relative L2): operator application <= 1e-5 vs the reference CPU
path (the oracle with the reference's kernels, or its restatement), and the
two FFT forms within 2e-6 of each other.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

OP_TOL = 1e-5
FORMS_TOL = 2e-6


def _ts_sense(pg, n, M, L, nc, seed, nz=1):
    from powergrid_b200 import synthetic as S
    rng = S.Rng(seed)
    inter = max(1, M // 2048)
    if nz == 1:
        kx, ky, t = S.spiral(n, inter, M // inter, 10e-3)
        kz = np.zeros_like(kx)
    else:
        kx, ky, kz, t = S.stack_of_spirals(n, nz, inter, M // inter, 10e-3)
    fm = S.field_map(rng, n, n, nz, 80.0)
    sm = S.coil_maps(rng, n, n, nz, nc)
    N = n * n * nz
    G = pg.Gnufft(kx.size, 2.0, n, n, nz, kx, ky, kz)
    A = pg.TimeSegmentation(G, fm, t, kx.size, N, L, 1, 1)
    Sg = pg.SENSE(A, sm, kx.size, N, nc)
    return (kx, ky, kz, t, fm, sm), (G, A, Sg)


def _cufft_form(build):
    old = os.environ.get("PG_CUFFT")
    os.environ["PG_CUFFT"] = "1"
    try:
        return build()
    finally:
        if old is None:
            del os.environ["PG_CUFFT"]
        else:
            os.environ["PG_CUFFT"] = old


@pytest.mark.parametrize("n", [32, 64, 128, 256, 512])
def test_own_fft_passes_match_cufft(pg, n):
    """Forward and adjoint of SENSE<TS<Gnufft>> (L=4, 2 coils) with the own FFT
    passes and with cuFFT, at grids 64^2 ... 1024^2."""
    from powergrid_b200 import synthetic as S
    M = 8192 if n <= 128 else 32768
    arrays, own = _ts_sense(pg, n, M, 4, 2, 40 + n)
    _, ref = _cufft_form(lambda: _ts_sense(pg, n, M, 4, 2, 40 + n))
    x = S.image(S.Rng(7), n * n)
    y1, y2 = own[2] * x, ref[2] * x
    e_f = rel_l2(y1, y2)
    a1, a2 = own[2] / y2, ref[2] / y2
    e_a = rel_l2(a1, a2)
    print(f"n={n}: forward {e_f:.2e}, adjoint {e_a:.2e}")
    assert e_f <= FORMS_TOL and e_a <= FORMS_TOL


@pytest.mark.parametrize("L,nc", [(1, 1), (4, 3), (8, 8)])
def test_fused_cluster_passes_equal_separate_passes(pg, L, nc):
    """The 256x256 grids' one-launch cluster form (rows in each CTA's shared
    memory, columns over distributed shared memory) against the separate
    passes: the same transforms in the same order (differences only from the
    compiler's fma contraction in each kernel), SENSE<TS<Gnufft>> 128^2 with
    batches of 1, 12 and 64 grids (the last more clusters than fit at once)."""
    from powergrid_b200 import synthetic as S
    _, own = _ts_sense(pg, 128, 8192, L, nc, 77)
    x = S.image(S.Rng(78), 128 * 128)
    y = own[2] * x
    xa = own[2] / y
    old = os.environ.get("PG_FFT_FUSED")
    os.environ["PG_FFT_FUSED"] = "0"
    try:
        y_sep = own[2] * x
        xa_sep = own[2] / y
    finally:
        if old is None:
            del os.environ["PG_FFT_FUSED"]
        else:
            os.environ["PG_FFT_FUSED"] = old
    e_f, e_a = rel_l2(y, y_sep), rel_l2(xa, xa_sep)
    print(f"fused vs separate, L={L}, {nc} coils: forward {e_f:.2e}, adjoint {e_a:.2e}")
    assert e_f <= 1e-6 and e_a <= 1e-6


@pytest.mark.parametrize("n", [128, 256])
def test_own_fft_passes_vs_reference(pg, oracle, n):
    """Gnufft 2-D against the reference CPU path at 256^2 and 512^2 grids."""
    from powergrid_b200 import synthetic as S
    kx, ky, t = S.spiral(n, 4, 2048, 10e-3)
    kz = np.zeros_like(kx)
    M = kx.size
    G = pg.Gnufft(M, 2.0, n, n, 1, kx, ky, kz)
    ref = oracle.gnufft(0, M, n, n, 1, kx, ky, kz)
    x = S.image(S.Rng(11), n * n)
    y = (S.image(S.Rng(12), M)).astype(np.complex64)
    e_f = rel_l2(G * x, ref.forward(x))
    e_a = rel_l2(G / y, ref.adjoint(y))
    print(f"n={n}: forward {e_f:.2e}, adjoint {e_a:.2e}")
    assert e_f <= OP_TOL and e_a <= OP_TOL


@pytest.mark.parametrize("n,nz", [(8, 8), (16, 32), (32, 16), (64, 8), (128, 64)])
def test_own_fft_passes_3d_match_cufft(pg, n, nz):
    """3-D SENSE<TS<Gnufft>> (L=3, 2 coils) with the own FFT passes and with
    cuFFT, from 16 x 16 x 16 up to the 256 x 256 x 128 grid of a 128^2 x 64
    volume; the z length differs from the in-plane one in most cases."""
    from powergrid_b200 import synthetic as S
    per_plane = 1024
    _, own = _ts_sense(pg, n, per_plane, 3, 2, 70 + n + nz, nz=nz)
    _, ref = _cufft_form(lambda: _ts_sense(pg, n, per_plane, 3, 2, 70 + n + nz, nz=nz))
    x = S.image(S.Rng(9), n * n * nz)
    y1, y2 = own[2] * x, ref[2] * x
    e_f = rel_l2(y1, y2)
    e_a = rel_l2(own[2] / y2, ref[2] / y2)
    print(f"{n}x{n}x{nz}: forward {e_f:.2e}, adjoint {e_a:.2e}")
    assert e_f <= FORMS_TOL and e_a <= FORMS_TOL


@pytest.mark.parametrize("n,nz", [(16, 8), (32, 16)])
def test_own_fft_passes_3d_vs_reference(pg, oracle, n, nz):
    """Gnufft 3-D on the own FFT passes against the reference CPU path."""
    from powergrid_b200 import synthetic as S
    kx, ky, kz, t = S.stack_of_spirals(n, nz, 2, 256, 5e-3)
    M = kx.size
    G = pg.Gnufft(M, 2.0, n, n, nz, kx, ky, kz)
    ref = oracle.gnufft(0, M, n, n, nz, kx, ky, kz)
    x = S.image(S.Rng(13), n * n * nz)
    y = S.image(S.Rng(14), M)
    e_f = rel_l2(G * x, ref.forward(x))
    e_a = rel_l2(G / y, ref.adjoint(y))
    print(f"{n}x{n}x{nz}: forward {e_f:.2e}, adjoint {e_a:.2e}")
    assert e_f <= OP_TOL and e_a <= OP_TOL


def _edge_case(kind, n):
    rng = np.random.default_rng(3)
    if kind == "border":          # samples on the -N/2 edge and just inside +N/2
        k = np.linspace(-n / 2, n / 2 - 1e-3, 64).astype(np.float32)
        kx = np.concatenate([np.full(64, -n / 2, np.float32), k])
        ky = np.concatenate([k, np.full(64, -n / 2, np.float32)])
    elif kind == "single":
        kx = np.array([3.25], np.float32)
        ky = np.array([-7.5], np.float32)
    else:                         # every sample in one tile: a dense cluster
        kx = (rng.random(3000) * 2.0 - 1.0).astype(np.float32)
        ky = (rng.random(3000) * 2.0 - 1.0).astype(np.float32)
    return kx, ky, np.zeros_like(kx)


@pytest.mark.parametrize("kind", ["border", "single", "cluster"])
def test_gridding_edge_cases_vs_reference(pg, oracle, kind):
    from powergrid_b200 import synthetic as S
    n = 32
    kx, ky, kz = _edge_case(kind, n)
    M = kx.size
    G = pg.Gnufft(M, 2.0, n, n, 1, kx, ky, kz)
    ref = oracle.gnufft(0, M, n, n, 1, kx, ky, kz)
    x = S.image(S.Rng(5), n * n)
    y = S.image(S.Rng(6), M)
    e_f = rel_l2(G * x, ref.forward(x))
    e_a = rel_l2(G / y, ref.adjoint(y))
    print(f"{kind}: forward {e_f:.2e}, adjoint {e_a:.2e}")
    assert e_f <= OP_TOL and e_a <= OP_TOL


def test_adjoint_of_zero_data_is_zero(pg):
    from powergrid_b200 import synthetic as S
    n = 64
    kx, ky, t = S.spiral(n, 2, 1024, 5e-3)
    G = pg.Gnufft(kx.size, 2.0, n, n, 1, kx, ky, np.zeros_like(kx))
    x = G / np.zeros(kx.size, np.complex64)
    assert np.all(x == 0)
