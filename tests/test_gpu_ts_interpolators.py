"""TimeSegmentation with the min-max (interptype 2, TimeSegmentation.cpp:94-156)
and histogram (interptype 3, :157-211) interpolators.

Their tables come from inverting Toeplitz Gram matrices of exponentials whose
condition number grows fast with L; the library builds them in double
precision, the reference in float.  The reference's float path agrees with
FP64 to 1e-5 only for small L (L = 3 at +-100 Hz here; 0.09-0.3 relative
error at L = 4-6), so every case is checked (<= 1e-5 relative L2 per operator
application) against the reference CPU path with its table built in double
(the restated float gridding, table rounded from double), states its FP64
error (no larger than that path's own, + 1e-5), and is checked against the
all-float reference path where that path is itself within 1e-4 of FP64.
The dense tables (every sample weights every segment) run through the fused
gridding in 2-D (up to 8 segments per sample) and one segment at a time in
3-D, as the reference applies them.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _case(dim):
    from powergrid_b200 import synthetic as S
    if dim == 2:
        n, nz = 32, 1
        kx, ky, t = S.spiral(n, 4, 1024, 8e-3)
        kz = np.zeros_like(kx)
    else:
        n, nz = 16, 4
        kx, ky, kz, t = S.stack_of_spirals(n, nz, 2, 256, 8e-3)
    fm = S.field_map(S.Rng(61), n, n, nz, 100.0)
    return n, nz, kx, ky, kz, t, fm


@pytest.mark.parametrize("dim,L,typ", [(2, 3, 2), (2, 3, 3), (2, 4, 2), (2, 4, 3), (2, 6, 2), (3, 4, 2), (3, 4, 3)])
def test_minmax_interpolators_vs_fp64(pg, oracle, dim, L, typ):
    from powergrid_b200 import synthetic as S
    n, nz, kx, ky, kz, t, fm = _case(dim)
    M, N = kx.size, n * n * nz
    G = pg.Gnufft(M, 2.0, n, n, nz, kx, ky, kz)
    A = pg.TimeSegmentation(G, fm, t, M, N, L, typ, 1)
    R32 = oracle.gnufft(0, M, n, n, nz, kx, ky, kz)
    R64 = oracle.gnufft(1, M, n, n, nz, kx, ky, kz)
    T32 = oracle.timeseg(R32, fm, t, M, N, L, typ)                  # all float (the reference)
    T32d = oracle.timeseg(R32, fm, t, M, N, L, typ, tables64=True)  # float gridding, double table
    T64 = oracle.timeseg(R64, fm, t, M, N, L, typ)
    x = S.image(S.Rng(62), N)
    d = S.image(S.Rng(63), M)
    y, xa = A * x, A / d
    yd, xd = T32d.forward(x), T32d.adjoint(d)
    y64, x64 = T64.forward(x.astype(np.complex128)), T64.adjoint(d.astype(np.complex128))
    y32, x32 = T32.forward(x), T32.adjoint(d)
    ef, ea = rel_l2(y, yd), rel_l2(xa, xd)
    rf, ra = rel_l2(y32, y64), rel_l2(x32, x64)
    print(f"dim {dim} L {L} type {typ}: fwd {ef:.2e} adj {ea:.2e} vs reference path with the double table "
          f"(fp64 {rel_l2(y, y64):.2e} / {rel_l2(xa, x64):.2e}, that path {rel_l2(yd, y64):.2e} / "
          f"{rel_l2(xd, x64):.2e}); all-float reference vs fp64 {rf:.2e} / {ra:.2e}")
    assert ef <= TOL and ea <= TOL
    assert rel_l2(y, y64) <= rel_l2(yd, y64) + TOL and rel_l2(xa, x64) <= rel_l2(xd, x64) + TOL
    if rf <= 1e-4 and ra <= 1e-4:
        assert rel_l2(y, y32) <= rf + TOL and rel_l2(xa, x32) <= ra + TOL


def test_minmax_sense_batched_matches_per_coil(pg):
    """SENSE over the dense 2-D table (fused, coils batched) equals coil-by-coil application."""
    from powergrid_b200 import synthetic as S
    n, nz, kx, ky, kz, t, fm = _case(2)
    M, N, nc = kx.size, n * n, 3
    sm = S.coil_maps(S.Rng(64), n, n, 1, nc)
    G = pg.Gnufft(M, 2.0, n, n, 1, kx, ky, kz)
    A = pg.TimeSegmentation(G, fm, t, M, N, 4, 2, 1)
    Sg = pg.SENSE(A, sm, M, N, nc)
    x = S.image(S.Rng(65), N)
    y = Sg * x
    smr = sm.reshape(nc, N)
    ref = np.concatenate([A * (smr[c] * x).astype(np.complex64) for c in range(nc)])
    assert rel_l2(y, ref) <= 2e-6
