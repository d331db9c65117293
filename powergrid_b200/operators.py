"""Python mirror of PowerGrid's operator API over the sm_100a C ABI.

Names, constructor arguments and operator semantics follow the reference:

    G = Gnufft(dataLength, gridos, nx, ny, nz, kx, ky, kz, ix, iy, iz)   # Gnufft.h:51-53
    A = TimeSegmentation(G, fieldMap, tvec, n1, n2, L, interptype, shots) # TimeSegmentation.h:70-71
    S = SENSE(A, senseMap, n1, n2, nc)                                   # SENSE.h:64
    y = S * x        # operator*  (forward)
    x = S / y        # operator/  (adjoint)
    x = reconSolve(data, S, QuadPenalty(nx, ny, nz, beta), kx, ky, kz, nx, ny, nz, tvec, niter)

Vectors are numpy complex64 (host) — or CUDA torch tensors, which stay on
the device.  Composites hold a reference to the operator they wrap
(the reference keeps a raw pointer and leaves lifetime to the caller,
SENSE.cpp:39).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import P, U64, Penalty, check

__all__ = ["Gnufft", "Gdft", "GdftR2", "TimeSegmentation", "SENSE", "pcSenseTimeSeg", "pcSENSE", "LRobj", "QuadPenalty",
           "TVPenalty", "R_lowRank", "pcg_state_save", "pcg_resume",
           "calc3DDensityCompensation", "gridCoilImages", "calcSumOfSquaresImage", "solve_pwls_pcg", "reconSolve",
           "init"]


def init(device: int = 0) -> None:
    check(_lib.load().pg_init(device))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _c64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex64))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(P)


def _is_torch(v) -> bool:
    return type(v).__module__.startswith("torch")


def _stream_ptr(stream):
    if stream is None:
        import torch
        return P(torch.cuda.current_stream().cuda_stream)
    return P(getattr(stream, "cuda_stream", stream))


class _Op:
    """Common operator behaviour: operator* / operator/ and shapes."""

    def __init__(self, handle: P, keep=()):
        self._h = handle
        self._keep = list(keep)
        nd, ni = U64(), U64()
        check(_lib.load().pg_op_shape(self._h, C.byref(nd), C.byref(ni)))
        self.n_data, self.n_image = int(nd.value), int(ni.value)

    @property
    def handle(self):
        return self._h

    def forward(self, x, out=None, stream=None):
        if _is_torch(x):
            import torch
            y = out if out is not None else torch.empty(self.n_data, dtype=torch.complex64, device=x.device)
            check(_lib.load().pg_op_forward_device(self._h, P(x.data_ptr()), P(y.data_ptr()), _stream_ptr(stream)))
            return y
        x = _c64(x)
        if x.size != self.n_image:
            raise ValueError(f"operator*: expected {self.n_image} image elements, got {x.size}")
        y = np.empty(self.n_data, dtype=np.complex64)
        check(_lib.load().pg_op_forward(self._h, _ptr(x), _ptr(y)))
        return y

    def adjoint(self, y, out=None, stream=None):
        if _is_torch(y):
            import torch
            x = out if out is not None else torch.empty(self.n_image, dtype=torch.complex64, device=y.device)
            check(_lib.load().pg_op_adjoint_device(self._h, P(y.data_ptr()), P(x.data_ptr()), _stream_ptr(stream)))
            return x
        y = _c64(y)
        if y.size != self.n_data:
            raise ValueError(f"operator/: expected {self.n_data} data elements, got {y.size}")
        x = np.empty(self.n_image, dtype=np.complex64)
        check(_lib.load().pg_op_adjoint(self._h, _ptr(y), _ptr(x)))
        return x

    __mul__ = forward
    __truediv__ = adjoint

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().pg_op_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Gnufft(_Op):
    """Gridding NUFFT, Kaiser-Bessel width 4, oversampling gridos (Gnufft.cpp:34-122).

    ix/iy/iz are accepted for interface compatibility; the reference stores
    them without using them in the transform (Gnufft.cpp:47-49).
    """

    def __init__(self, dataLength, gridos, nx, ny, nz, kx, ky, kz, ix=None, iy=None, iz=None):
        kx, ky, kz = _f32(kx), _f32(ky), _f32(kz)
        h = P()
        check(_lib.load().pg_gnufft_create(C.byref(h), int(dataLength), float(gridos), int(nx), int(ny), int(nz),
                                            _ptr(kx), _ptr(ky), _ptr(kz)))
        self.Nx, self.Ny, self.Nz = int(nx), int(ny), int(nz)
        super().__init__(h)

    def binning(self):
        """(bin key per sample, sorted order, number of bins) of the device binning."""
        keys = np.zeros(self.n_data, np.uint32)
        perm = np.zeros(self.n_data, np.uint32)
        nb = U64()
        check(_lib.load().pg_util_gnufft_binning(self._h, _ptr(keys), _ptr(perm), C.byref(nb)))
        return keys, perm, int(nb.value)

    @property
    def grid_length(self) -> int:
        """Cells of the oversampled grid (Gnufft.cpp:56-61)."""
        n = U64()
        check(_lib.load().pg_gnufft_grid_length(self._h, C.byref(n)))
        return int(n.value)

    def forwardSpatialInterp(self, grid):
        """Samples interpolated from an oversampled grid in the reference's layout (Gnufft.cpp:213-258)."""
        g = _c64(grid)
        if g.size != self.grid_length:
            raise ValueError(f"grid has {g.size} cells, expected {self.grid_length}")
        out = np.empty(self.n_data, np.complex64)
        check(_lib.load().pg_gnufft_forward_spatial_interp(self._h, _ptr(g), _ptr(out)))
        return out

    def adjointSpatialInterp(self, data):
        """Samples spread onto the oversampled grid, no FFT (Gnufft.cpp:261-330)."""
        d = _c64(data)
        if d.size != self.n_data:
            raise ValueError(f"data has {d.size} samples, expected {self.n_data}")
        out = np.empty(self.grid_length, np.complex64)
        check(_lib.load().pg_gnufft_adjoint_spatial_interp(self._h, _ptr(d), _ptr(out)))
        return out


class Gdft(_Op):
    """Exact field-corrected DFT (Gdft.cpp:33-136); FM in rad/s, t in s."""

    def __init__(self, nk, ni, kx, ky, kz, ix, iy, iz, FM, t):
        a = [_f32(v) for v in (kx, ky, kz, ix, iy, iz, FM, t)]
        h = P()
        check(_lib.load().pg_gdft_create(C.byref(h), int(nk), int(ni), *[_ptr(v) for v in a]))
        super().__init__(h)


class GdftR2(_Op):
    """Field-corrected DFT with field-map gradient (through-voxel dephasing) factors
    (GdftR2.cpp:32-150, ftCpuWithGrads.cpp:93-216); FM in rad/s, t in s."""

    def __init__(self, nk, ni, kx, ky, kz, ix, iy, iz, FM, t, num_x, num_y, num_z):
        a = [_f32(v) for v in (kx, ky, kz, ix, iy, iz, FM, t)]
        h = P()
        check(_lib.load().pg_gdftr2_create(C.byref(h), int(nk), int(ni), *[_ptr(v) for v in a], int(num_x),
                                            int(num_y), int(num_z)))
        super().__init__(h)


class TimeSegmentation(_Op):
    """Time-segmented field correction (TimeSegmentation.cpp:37-324); interptype 1 = Hanning."""

    def __init__(self, G: _Op, fieldMap, timeVec, n1, n2, L, interptype=1, shots=1):
        fm, tv = _f32(fieldMap), _f32(timeVec)
        h = P()
        check(_lib.load().pg_timeseg_create(C.byref(h), G.handle, _ptr(fm), _ptr(tv), int(n1), int(n2), int(L),
                                             int(interptype), int(shots)))
        super().__init__(h, keep=[G])


TimeSegmentation.binning = Gnufft.binning


class SENSE(_Op):
    """SENSE coil loop (SENSE.cpp:33-97); senseMap complex, n2*nc, coil-major."""

    def __init__(self, G: _Op, senseMap, n1, n2, nc):
        sm = _c64(senseMap)
        h = P()
        check(_lib.load().pg_sense_create(C.byref(h), G.handle, _ptr(sm), int(n1), int(n2), int(nc)))
        super().__init__(h, keep=[G])


class pcSenseTimeSeg(_Op):
    """Multishot phase-corrected SENSE over per-shot TimeSegmentation<Gnufft> (pcSenseTimeSeg.cpp:41-171)."""

    def __init__(self, kx, ky, kz, nx, ny, nz, nc, t, L, intType, SENSEmap, FieldMap, ShotPhaseMap):
        kx, ky, kz, t, fm, pm = (_f32(v) for v in (kx, ky, kz, t, FieldMap, ShotPhaseMap))
        sm = _c64(SENSEmap)
        h = P()
        check(_lib.load().pg_pcsense_timeseg_create(C.byref(h), _ptr(kx), _ptr(ky), _ptr(kz), kx.size, int(nx),
                                                     int(ny), int(nz), int(nc), _ptr(t), int(L), int(intType),
                                                     _ptr(sm), _ptr(fm), _ptr(pm), pm.size))
        super().__init__(h)


class pcSENSE(_Op):
    """Multishot phase-corrected SENSE over one Gdft per shot (pcSENSE.cpp:40-153).

    As in the reference, forward and adjoint both weight by exp(+i*ShotPhaseMap)
    (pcSENSE.cpp:103, 123, 146)."""

    def __init__(self, kx, ky, kz, nx, ny, nz, nc, t, SENSEmap, FieldMap, ShotPhaseMap):
        kx, ky, kz, t, fm, pm = (_f32(v) for v in (kx, ky, kz, t, FieldMap, ShotPhaseMap))
        sm = _c64(SENSEmap)
        h = P()
        check(_lib.load().pg_pcsense_create(C.byref(h), _ptr(kx), _ptr(ky), _ptr(kz), kx.size, int(nx), int(ny),
                                             int(nz), int(nc), _ptr(t), _ptr(sm), _ptr(fm), _ptr(pm), pm.size))
        super().__init__(h)


def _basis(v, rank, n_img):
    """A rank x n_img complex basis as a column-major complex64 array."""
    v = np.asarray(v, dtype=np.complex64)
    if v.shape != (rank, n_img):
        v = v.reshape(rank, n_img, order="F")
    return np.ascontiguousarray(v.reshape(-1, order="F"))


class LRobj(_Op):
    """Partial-separability model (lowRank/LRobj.cpp:27-68): x = vec(X) with X
    NimgSize x n_rank; image i = column i of X * vBasis goes through All[i].
    The per-image operators are borrowed (kept alive by this object)."""

    def __init__(self, NimgSize, N_data, n_rank, n_img, vBasis, All):
        ops = list(All)
        if len(ops) != int(n_img):
            raise ValueError(f"LRobj: {len(ops)} operators for {n_img} images")
        self.v = _basis(vBasis, int(n_rank), int(n_img))
        hs = (P * len(ops))(*[o.handle for o in ops])
        h = P()
        check(_lib.load().pg_lowrank_create(C.byref(h), int(NimgSize), int(N_data), int(n_rank), int(n_img),
                                             _ptr(self.v), C.cast(hs, P)))
        super().__init__(h, keep=ops)


class R_lowRank:
    """Low-rank wrapper of a QuadPenalty/TVPenalty (lowRank/R_lowRank.cpp:27-95):
    R applied to the columns of X * vBasis^H.  As in the reference the
    gradient is defined only for rank == nImages and comes back rank-fastest,
    and Denom carries beta twice."""

    def __init__(self, R1, rank, nImages, vBasis):
        self.R, self.rank, self.n_img = R1, int(rank), int(nImages)
        self.v = _basis(vBasis, self.rank, self.n_img)

    def Gradient(self, x):
        import torch
        g = torch.empty_like(x)
        pen = self.R._struct()
        check(_lib.load().pg_lowrank_penalty_gradient_device(C.byref(pen), self.rank, self.n_img, _ptr(self.v),
                                                              P(x.data_ptr()), P(g.data_ptr()), _stream_ptr(None)))
        return g

    def Denom(self, ddir, x) -> float:
        import torch
        torch.cuda.current_stream().synchronize()
        out = C.c_double()
        pen = self.R._struct()
        check(_lib.load().pg_lowrank_penalty_denom_device(C.byref(pen), self.rank, self.n_img, _ptr(self.v),
                                                           P(ddir.data_ptr()), P(x.data_ptr()), C.byref(out)))
        return out.value


def calc3DDensityCompensation(kx, ky, kz, Ninplane, Nz):
    """Sample density compensation (reconSupport/directRecon.cpp:28-61): two Pipe
    iterations on a 3x oversampled grid, |dcf| normalised to unit L2 norm."""
    kx, ky, kz = _f32(kx), _f32(ky), _f32(kz)
    out = np.empty(kx.size, np.float32)
    check(_lib.load().pg_density_compensation(_ptr(kx), _ptr(ky), _ptr(kz), kx.size, int(Ninplane), int(Nz),
                                              _ptr(out)))
    return out


def gridCoilImages(G: Gnufft, dcf, data, Ncoils):
    """Per-coil gridded images G / (dcf .* data_c) (directRecon.cpp:108-133), coil-major."""
    w = _f32(dcf)
    d = _c64(data)
    nc = int(Ncoils)
    if w.size != G.n_data or d.size != G.n_data * nc:
        raise ValueError("dcf / data sizes do not match the operator")
    out = np.empty(G.n_image * nc, np.complex64)
    check(_lib.load().pg_grid_coil_images(G.handle, _ptr(w), _ptr(d), nc, _ptr(out)))
    return out


def calcSumOfSquaresImage(coilImages, Ncoils):
    """sqrt(sum_c |img_c|) per voxel (directRecon.cpp:63-73; a sum of magnitudes, as the reference has it)."""
    img = _c64(coilImages)
    nc = int(Ncoils)
    if img.size % nc:
        raise ValueError("coil images not divisible by Ncoils")
    out = np.empty(img.size // nc, np.float32)
    check(_lib.load().pg_sum_of_squares_image(_ptr(img), img.size // nc, nc, _ptr(out)))
    return out


class QuadPenalty:
    """Quadratic roughness penalty (QuadPenalty.h:43)."""
    kind = 0

    def __init__(self, nx, ny, nz, beta, dims2penalize=3):
        self.nx, self.ny, self.nz, self.beta, self.dims2penalize = int(nx), int(ny), int(nz), float(beta), int(
            dims2penalize)
        self.delta = 1.0

    def _struct(self) -> Penalty:
        return Penalty(self.kind, self.nx, self.ny, self.nz, self.beta, self.delta, self.dims2penalize)

    def Gradient(self, x):
        import torch
        g = torch.empty_like(x)
        pen = self._struct()
        check(_lib.load().pg_penalty_gradient_device(C.byref(pen), P(x.data_ptr()), P(g.data_ptr()),
                                                      _stream_ptr(None)))
        return g

    def Denom(self, ddir, x) -> float:
        out = C.c_double()
        pen = self._struct()
        import torch
        torch.cuda.current_stream().synchronize()
        check(_lib.load().pg_penalty_denom_device(C.byref(pen), P(ddir.data_ptr()), P(x.data_ptr()), C.byref(out)))
        return out.value


class TVPenalty(QuadPenalty):
    """Total-variation penalty with smoothing delta (TVPenalty.h:42)."""
    kind = 1

    def __init__(self, nx, ny, nz, beta, delta, dims2penalize=3):
        super().__init__(nx, ny, nz, beta, dims2penalize)
        self.delta = float(delta)


def solve_pwls_pcg(xInitial, A: _Op, W, yi, R: QuadPenalty, niter):
    """PWLS conjugate gradient (solve_pwls_pcg.hpp:48-167) on the device.

    Host arrays in, host array out; xInitial/W may be None (zeros / ones).
    Returns (x, iterations_completed).
    """
    yi = _c64(yi)
    x = np.empty(A.n_image, dtype=np.complex64)
    x0 = None if xInitial is None else _c64(xInitial)
    Wa = None if W is None else _f32(W)
    it = U64()
    if isinstance(R, R_lowRank):
        pen = R.R._struct()
        check(_lib.load().pg_pcg_solve_lowrank(A.handle, None if x0 is None else _ptr(x0),
                                                None if Wa is None else _ptr(Wa), _ptr(yi), C.byref(pen), R.rank,
                                                R.n_img, _ptr(R.v), int(niter), _ptr(x), C.byref(it)))
        return x, int(it.value)
    pen = R._struct()
    check(_lib.load().pg_pcg_solve(A.handle, None if x0 is None else _ptr(x0), None if Wa is None else _ptr(Wa),
                                    _ptr(yi), C.byref(pen), int(niter), _ptr(x), C.byref(it)))
    return x, int(it.value)


def solve_pwls_pcg_device(A: _Op, yi, R: QuadPenalty, niter, x_out, xInitial=None, W=None, iters=None, stream=None):
    """Device-resident solve on torch CUDA tensors (stream-ordered)."""
    pen = R._struct()
    check(_lib.load().pg_pcg_solve_device(A.handle, None if xInitial is None else P(xInitial.data_ptr()),
                                           None if W is None else P(W.data_ptr()), P(yi.data_ptr()), C.byref(pen),
                                           int(niter), P(x_out.data_ptr()),
                                           None if iters is None else P(iters.data_ptr()), _stream_ptr(stream)))
    return x_out


def pcg_state_save(A: _Op) -> bytes:
    """The solver state on A after a solve (x, Ax, residual, direction(s), scalars, counters)."""
    n = U64()
    check(_lib.load().pg_pcg_state_size(A.handle, C.byref(n)))
    buf = np.empty(n.value, np.uint8)
    check(_lib.load().pg_pcg_state_save(A.handle, _ptr(buf), n.value))
    return buf.tobytes()


def pcg_resume(A: _Op, state: bytes, W, yi, R: QuadPenalty, niter):
    """Load `state` onto A and run niter more PCG iterations; returns (x, iterations counted from the start)."""
    buf = np.frombuffer(state, np.uint8).copy()
    pen = R._struct()
    check(_lib.load().pg_pcg_state_load(A.handle, C.byref(pen), _ptr(buf), buf.size))
    yi = _c64(yi)
    Wa = None if W is None else _f32(W)
    x = np.empty(A.n_image, dtype=np.complex64)
    it = U64()
    check(_lib.load().pg_pcg_resume(A.handle, None if Wa is None else _ptr(Wa), _ptr(yi), C.byref(pen), int(niter),
                                     _ptr(x), C.byref(it)))
    return x, int(it.value)


def reconSolve(data, Sg: _Op, R: QuadPenalty, kx=None, ky=None, kz=None, Nx=None, Ny=None, Nz=None, tvec=None,
               niter=10):
    """reconSolve (reconSolve.h:63-82): W = 1, x0 = 0."""
    x, _ = solve_pwls_pcg(None, Sg, None, data, R, niter)
    return x
