"""ORACLE / TEST INFRASTRUCTURE ONLY — the checker, never the product.

ctypes front end of the CPU oracle (oracle_capi.cpp over pg_oracle.hpp):
a restatement of PowerGrid's system-operator path in float (the reference
CPU path) and double (the FP64 oracle), optionally running Gnufft/Gdft on
the reference's own kernels compiled from its sources (oracle/_ref/).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libpgref.so")

F32, F64, C64, C128 = np.float32, np.float64, np.complex64, np.complex128
P = C.c_void_p
U64 = C.c_uint64

_lib = None


def build(ref: bool = False) -> None:
    """Compile the restatement (and, where the reference tree exists, its kernels)."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_last_error.restype = C.c_char_p
        L.orc_gnufft_new.restype = P
        L.orc_gnufft_new.argtypes = [C.c_int, U64, C.c_float, U64, U64, U64, P, P, P]
        L.orc_gdft_new.restype = P
        L.orc_gdft_new.argtypes = [C.c_int, U64, U64] + [P] * 8
        L.orc_gdftr2_new.restype = P
        L.orc_gdftr2_new.argtypes = [C.c_int, U64, U64] + [P] * 8 + [U64, U64, U64]
        L.orc_timeseg_new.restype = P
        L.orc_timeseg_new.argtypes = [P, P, P, U64, U64, U64, U64, U64, C.c_int]
        L.orc_sense_new.restype = P
        L.orc_sense_new.argtypes = [P, P, U64, U64, U64]
        L.orc_pcsense_ts_new.restype = P
        L.orc_pcsense_ts_new.argtypes = [C.c_int, P, P, P, U64, U64, U64, U64, U64, P, U64, U64, P, P, P, U64]
        L.orc_pcsense_new.restype = P
        L.orc_pcsense_new.argtypes = [C.c_int, P, P, P, U64, U64, U64, U64, U64, P, P, P, P, U64]
        L.orc_gnufft_grid_len.restype = U64
        L.orc_gnufft_grid_len.argtypes = [P]
        L.orc_gnufft_interp_fwd.argtypes = [P, P, P]
        L.orc_gnufft_interp_adj.argtypes = [P, P, P]
        L.orc_density_compensation.argtypes = [C.c_int, P, P, P, U64, U64, U64, P]
        L.orc_free.argtypes = [P]
        L.orc_data_len.restype = U64
        L.orc_data_len.argtypes = [P]
        L.orc_image_len.restype = U64
        L.orc_image_len.argtypes = [P]
        L.orc_forward.argtypes = [P, P, P]
        L.orc_adjoint.argtypes = [P, P, P]
        L.orc_pcg.argtypes = [P, P, P, P, C.c_int, U64, U64, U64, C.c_double, C.c_double, U64, U64, P]
        L.orc_pcg_fp64_over_f32.argtypes = [P, P, P, C.c_int, U64, U64, U64, C.c_double, C.c_double, U64, U64, P]
        L.orc_penalty_gradient.argtypes = [C.c_int, C.c_int, U64, U64, U64, C.c_double, C.c_double, U64, P, P]
        L.orc_penalty_denom.argtypes = [C.c_int, C.c_int, U64, U64, U64, C.c_double, C.c_double, U64, P, P, P]
        L.orc_lowrank_new.restype = P
        L.orc_lowrank_new.argtypes = [U64, U64, U64, U64, P, P]
        L.orc_pcg_lowrank.argtypes = [P, P, P, P, C.c_int, U64, U64, U64, C.c_double, C.c_double, U64, U64, P, U64,
                                      P]
        L.orc_lowrank_gradient.argtypes = [C.c_int, C.c_int, U64, U64, U64, C.c_double, C.c_double, U64, U64, P, P,
                                           P]
        L.orc_lowrank_denom.argtypes = [C.c_int, C.c_int, U64, U64, U64, C.c_double, C.c_double, U64, U64, P, P, P,
                                        P]
        L.orc_kb_lut.argtypes = [C.c_int, C.c_float, P, U64, P]
        L.orc_timeseg_tables.argtypes = [P, P, P, P, P]
        L.orc_fft.argtypes = [C.c_int, P, P, C.c_int, C.c_int]
        L.orc_use_reference.argtypes = [C.c_char_p]
        L.orc_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def reference_available() -> bool:
    return os.path.exists(REF_PATH)


def use_reference(on: bool = True) -> None:
    """Route Gnufft/Gdft (float, double) through the reference's compiled kernels."""
    rc = lib().orc_use_reference(REF_PATH.encode() if on else None)
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def _p(a: np.ndarray):
    return a.ctypes.data_as(P)


def _f32(a):
    return np.ascontiguousarray(a, dtype=F32)


class Op:
    """An oracle operator: forward = operator*, adjoint = operator/."""

    def __init__(self, handle, prec: int, keep=()):
        if not handle:
            raise RuntimeError("oracle: " + lib().orc_last_error().decode())
        self.h = handle
        self.prec = prec
        self._keep = list(keep)

    @property
    def cdtype(self):
        return C64 if self.prec == 0 else C128

    @property
    def rdtype(self):
        return F32 if self.prec == 0 else F64

    @property
    def n_data(self) -> int:
        return int(lib().orc_data_len(self.h))

    @property
    def n_image(self) -> int:
        return int(lib().orc_image_len(self.h))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=self.cdtype)
        y = np.zeros(self.n_data, dtype=self.cdtype)
        lib().orc_forward(self.h, _p(x), _p(y))
        return y

    def adjoint(self, y: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=self.cdtype)
        x = np.zeros(self.n_image, dtype=self.cdtype)
        lib().orc_adjoint(self.h, _p(y), _p(x))
        return x

    __mul__ = forward
    __truediv__ = adjoint

    def pcg(self, y, penalty: str, nx, ny, nz, beta, delta=1.0, dims2pen=3, niter=10, x0=None, W=None):
        y = np.ascontiguousarray(y, dtype=self.cdtype)
        x = np.zeros(self.n_image, dtype=self.cdtype)
        x0p = None if x0 is None else _p(np.ascontiguousarray(x0, dtype=self.cdtype))
        Wa = None if W is None else np.ascontiguousarray(W, dtype=self.rdtype)
        kind = {"quad": 0, "tv": 1}[penalty]
        n = lib().orc_pcg(self.h, x0p, None if Wa is None else _p(Wa), _p(y), kind, nx, ny, nz, beta, delta,
                          dims2pen, niter, _p(x))
        return x, n

    def pcg_fp64_solver(self, y, penalty: str, nx, ny, nz, beta, delta=1.0, dims2pen=3, niter=10, W=None):
        """PWLS-PCG with FP64 vectors, inner products and steps over this float
        operator (inputs rounded to float, outputs widened): the operator's FP32
        rounding is then the solve's only FP32 step.  Returns complex128."""
        if self.prec != 0:
            raise ValueError("pcg_fp64_solver needs a float (precision 0) operator")
        y = np.ascontiguousarray(y, dtype=C128)
        x = np.zeros(self.n_image, dtype=C128)
        Wa = None if W is None else np.ascontiguousarray(W, dtype=F64)
        n = lib().orc_pcg_fp64_over_f32(self.h, None if Wa is None else _p(Wa), _p(y), {"quad": 0, "tv": 1}[penalty],
                                        nx, ny, nz, beta, delta, dims2pen, niter, _p(x))
        if n < 0:
            raise RuntimeError("oracle: " + lib().orc_last_error().decode())
        return x, n

    def timeseg_tables(self):
        L = int(lib().orc_timeseg_tables(self.h, None, None, None, _p(np.zeros(2))))
        n1, n2 = self.n_data, self.n_image
        AA = np.zeros(n1 * L, self.cdtype)
        Wo = np.zeros(n2 * (L + 1) if L > 1 else n2, self.cdtype)
        WoH = np.zeros_like(Wo)
        tt = np.zeros(2)
        lib().orc_timeseg_tables(self.h, _p(AA), _p(Wo), _p(WoH), _p(tt))
        return AA.reshape(L, n1), Wo, WoH, tt

    def __del__(self):
        try:
            if _lib is not None and self.h:
                _lib.orc_free(self.h)
        except Exception:
            pass


def gnufft(prec, M, nx, ny, nz, kx, ky, kz, gridos=2.0) -> Op:
    kx, ky, kz = _f32(kx), _f32(ky), _f32(kz)
    return Op(lib().orc_gnufft_new(prec, M, gridos, nx, ny, nz, _p(kx), _p(ky), _p(kz)), prec)


def gdft(prec, kx, ky, kz, ix, iy, iz, fm, t) -> Op:
    a = [_f32(v) for v in (kx, ky, kz, ix, iy, iz, fm, t)]
    return Op(lib().orc_gdft_new(prec, a[0].size, a[3].size, *[_p(v) for v in a]), prec)


def gdftr2(prec, kx, ky, kz, ix, iy, iz, fm, t, nx, ny, nz) -> Op:
    """GdftR2 (GdftR2.cpp:32-150); prec 2 = FP64 DFT and sinc."""
    a = [_f32(v) for v in (kx, ky, kz, ix, iy, iz, fm, t)]
    return Op(lib().orc_gdftr2_new(prec, a[0].size, a[3].size, *[_p(v) for v in a], nx, ny, nz), prec)


def timeseg(G: Op, fm, t, n1, n2, L, interptype=1, shots=1, tables64=False) -> Op:
    """TimeSegmentation over G; tables64 builds the min-max / histogram table in
    double and rounds it (float G only)."""
    fm, t = _f32(fm), _f32(t)
    return Op(lib().orc_timeseg_new(G.h, _p(fm), _p(t), n1, n2, L, interptype, shots, int(tables64)), G.prec,
              keep=[G])


def sense(G: Op, smap, n1, n2, nc) -> Op:
    s = np.ascontiguousarray(smap, dtype=C64)
    return Op(lib().orc_sense_new(G.h, _p(s), n1, n2, nc), G.prec, keep=[G])


def pcsense_timeseg(prec, kx, ky, kz, nx, ny, nz, nc, t, L, smap, fm, pmap, interptype=1) -> Op:
    kx, ky, kz, t, fm, pm = (_f32(v) for v in (kx, ky, kz, t, fm, pmap))
    s = np.ascontiguousarray(smap, dtype=C64)
    return Op(lib().orc_pcsense_ts_new(prec, _p(kx), _p(ky), _p(kz), kx.size, nx, ny, nz, nc, _p(t), L, interptype,
                                       _p(s), _p(fm), _p(pm), pm.size), prec)


def pcsense(prec, kx, ky, kz, nx, ny, nz, nc, t, smap, fm, pmap) -> Op:
    """pcSENSE over per-shot Gdft (pcSENSE.cpp:40-153); prec 2 = FP64 DFT."""
    kx, ky, kz, t, fm, pm = (_f32(v) for v in (kx, ky, kz, t, fm, pmap))
    s = np.ascontiguousarray(smap, dtype=C64)
    return Op(lib().orc_pcsense_new(prec, _p(kx), _p(ky), _p(kz), kx.size, nx, ny, nz, nc, _p(t), _p(s), _p(fm),
                                    _p(pm), pm.size), prec)


def forward_spatial_interp(G: Op, grid) -> np.ndarray:
    """Gnufft::forwardSpatialInterp (Gnufft.cpp:213-258) of a Gnufft oracle handle."""
    dt = C64 if G.prec == 0 else np.complex128
    g = np.ascontiguousarray(grid, dtype=dt)
    assert g.size == lib().orc_gnufft_grid_len(G.h)
    out = np.zeros(lib().orc_data_len(G.h), dtype=dt)
    lib().orc_gnufft_interp_fwd(G.h, _p(g), _p(out))
    return out


def adjoint_spatial_interp(G: Op, d) -> np.ndarray:
    """Gnufft::adjointSpatialInterp (Gnufft.cpp:261-330) of a Gnufft oracle handle."""
    dt = C64 if G.prec == 0 else np.complex128
    v = np.ascontiguousarray(d, dtype=dt)
    out = np.zeros(lib().orc_gnufft_grid_len(G.h), dtype=dt)
    lib().orc_gnufft_interp_adj(G.h, _p(v), _p(out))
    return out


def density_compensation(prec, kx, ky, kz, ninplane, nz) -> np.ndarray:
    """calc3DDensityCompensation (reconSupport/directRecon.cpp:28-61)."""
    kx, ky, kz = (_f32(v) for v in (kx, ky, kz))
    out = np.zeros(kx.size, dtype=F32 if prec == 0 else F64)
    lib().orc_density_compensation(prec, _p(kx), _p(ky), _p(kz), kx.size, ninplane, nz, _p(out))
    return out


def sum_of_squares_image(coil_images, nc) -> np.ndarray:
    """calcSumOfSquaresImage (directRecon.cpp:63-73): sqrt of the coil-ordered float sum of |img_c|."""
    img = np.ascontiguousarray(coil_images, dtype=C64).reshape(nc, -1)
    acc = np.zeros(img.shape[1], dtype=F32)
    for c in range(nc):
        acc = (acc + np.abs(img[c]).astype(F32)).astype(F32)
    return np.sqrt(acc).astype(F32)


def kb_lut(prec: int, gridos: float = 2.0):
    out = np.zeros(100000, dtype=F32 if prec == 0 else F64)
    beta = np.zeros(1)
    n = lib().orc_kb_lut(prec, gridos, _p(out), out.size, _p(beta))
    return out[:n].copy(), float(beta[0])


def fft(a: np.ndarray, sign: int) -> np.ndarray:
    a = np.ascontiguousarray(a.copy())
    prec = 0 if a.dtype == C64 else 1
    dims = np.array(a.shape, dtype=np.uint64)
    lib().orc_fft(prec, _p(a), _p(dims), a.ndim, sign)
    return a


def penalty_gradient(prec, kind, nx, ny, nz, beta, delta, dims2pen, x):
    x = np.ascontiguousarray(x, dtype=C64 if prec == 0 else C128)
    g = np.zeros_like(x)
    lib().orc_penalty_gradient(prec, {"quad": 0, "tv": 1}[kind], nx, ny, nz, beta, delta, dims2pen, _p(x), _p(g))
    return g


def penalty_denom(prec, kind, nx, ny, nz, beta, delta, dims2pen, ddir, x):
    ct = C64 if prec == 0 else C128
    d = np.ascontiguousarray(ddir, dtype=ct)
    x = np.ascontiguousarray(x, dtype=ct)
    out = np.zeros(2)
    lib().orc_penalty_denom(prec, {"quad": 0, "tv": 1}[kind], nx, ny, nz, beta, delta, dims2pen, _p(d), _p(x),
                            _p(out))
    return complex(out[0], out[1])


def _basis(v, rank, nimg):
    """rank x nimg complex basis, column-major, as interleaved float32 pairs."""
    v = np.asarray(v, dtype=C64).reshape(rank, nimg, order="F")
    return np.ascontiguousarray(v.reshape(-1, order="F")).view(F32)


def lowrank(n_image, n_data, rank, nimg, v, ops) -> Op:
    """LRobj (lowRank/LRobj.cpp:27-68) over oracle operators (borrowed: kept alive here)."""
    vb = _basis(v, rank, nimg)
    hs = (C.c_void_p * nimg)(*[o.h for o in ops])
    h = lib().orc_lowrank_new(n_image, n_data, rank, nimg, _p(vb), C.cast(hs, C.c_void_p))
    return Op(h, ops[0].prec, keep=list(ops))


def pcg_lowrank(op: Op, y, penalty: str, nx, ny, nz, beta, rank, v, delta=1.0, dims2pen=3, niter=10, x0=None,
                W=None):
    """solve_pwls_pcg with R_lowRank (lowRank/R_lowRank.cpp:27-95); v: rank x rank basis."""
    y = np.ascontiguousarray(y, dtype=op.cdtype)
    x = np.zeros(op.n_image, dtype=op.cdtype)
    x0p = None if x0 is None else _p(np.ascontiguousarray(x0, dtype=op.cdtype))
    Wa = None if W is None else np.ascontiguousarray(W, dtype=op.rdtype)
    vb = _basis(v, rank, rank)
    n = lib().orc_pcg_lowrank(op.h, x0p, None if Wa is None else _p(Wa), _p(y), {"quad": 0, "tv": 1}[penalty], nx,
                              ny, nz, beta, delta, dims2pen, rank, _p(vb), niter, _p(x))
    return x, n


def lowrank_gradient(prec, kind, nx, ny, nz, beta, delta, dims2pen, rank, v, x):
    x = np.ascontiguousarray(x, dtype=C64 if prec == 0 else C128)
    g = np.zeros_like(x)
    lib().orc_lowrank_gradient(prec, {"quad": 0, "tv": 1}[kind], nx, ny, nz, beta, delta, dims2pen, rank,
                               _p(_basis(v, rank, rank)), _p(x), _p(g))
    return g


def lowrank_denom(prec, kind, nx, ny, nz, beta, delta, dims2pen, rank, v, ddir, x):
    ct = C64 if prec == 0 else C128
    d = np.ascontiguousarray(ddir, dtype=ct)
    x = np.ascontiguousarray(x, dtype=ct)
    out = np.zeros(2)
    lib().orc_lowrank_denom(prec, {"quad": 0, "tv": 1}[kind], nx, ny, nz, beta, delta, dims2pen, rank,
                            _p(_basis(v, rank, rank)), _p(d), _p(x), _p(out))
    return complex(out[0], out[1])


def build_problem_op(prob, prec: int) -> Op:
    """The operator a Problem describes, as the reference's drivers compose it
    (PowerGridIsmrmrd.cpp:244-264, PowerGridPcSenseTimeSeg.cpp)."""
    from powergrid_b200.synthetic import image_coords  # noqa: WPS433 (shared generator)
    M = prob.kx.size
    n = prob.nimg
    if prob.op == "pcsense_ts":
        return pcsense_timeseg(prec, prob.kx, prob.ky, prob.kz, prob.nx, prob.ny, prob.nz, prob.nc, prob.t, prob.L,
                               prob.smap, prob.fm, prob.pmap)
    if prob.op == "sense_gdft":
        ix, iy, iz = image_coords(prob.nx, prob.ny, prob.nz)
        G = gdft(prec, prob.kx, prob.ky, prob.kz, ix, iy, iz, prob.fm, prob.t)
        return sense(G, prob.smap, M, n, prob.nc)
    G = gnufft(prec, M, prob.nx, prob.ny, prob.nz, prob.kx, prob.ky, prob.kz)
    if prob.op == "sense_ts_nufft":
        A = timeseg(G, prob.fm, prob.t, M, n, prob.L)
        return sense(A, prob.smap, M, n, prob.nc)
    return sense(G, prob.smap, M, n, prob.nc)
