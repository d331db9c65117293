"""Generate the golden fixtures in tests/golden/*.npz.

The outputs come from the reference's OWN kernels — PowerGrid/gridding.cpp,
griddingSupport.cpp, ftCpu.cpp and fftCPU.cpp compiled unmodified from the
reference tree into oracle/_ref/libpgref.so (oracle/Makefile, target `ref`;
ftCpuWithGrads.cpp too, for GdftR2),
with the project FFT behind the FFTW API — driven by the oracle's restated
Armadillo layers (TimeSegmentation, SENSE, pcSenseTimeSeg, PCG).  FP64
outputs come from the reference's double instantiation (Gnufft) and the
FP64 DFT restatement.

Run where the reference tree exists:  python tests/golden/make_golden.py [case ...]
Inputs are seeded (powergrid_b200.synthetic), so the files are reproducible.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import oracle as O  # noqa: E402
from powergrid_b200 import synthetic as S  # noqa: E402


def small_cases():
    """Seeded small problems (seconds on one CPU core)."""
    cases = {}
    # 2-D Gnufft, 32x32, 4-interleave spiral x 256
    n = 32
    kx, ky, t = S.spiral(n, 4, 256, 4e-3)
    cases["nufft2d"] = dict(nx=n, ny=n, nz=1, kx=kx, ky=ky, kz=np.zeros_like(kx), t=t,
                            x=S.image(S.Rng(101), n * n))
    # 3-D Gnufft, 16x16x8 stack of spirals
    kx, ky, kz, t = S.stack_of_spirals(16, 8, 2, 128, 3e-3)
    cases["nufft3d"] = dict(nx=16, ny=16, nz=8, kx=kx, ky=ky, kz=kz, t=t, x=S.image(S.Rng(102), 16 * 16 * 8))
    # 3-D Gdft, 8x8x4 image, 512 samples, +-150 Hz
    kx, ky, kz, t = S.stack_of_spirals(8, 4, 2, 64, 25e-3)
    cases["gdft3d"] = dict(nx=8, ny=8, nz=4, kx=kx, ky=ky, kz=kz, t=t, x=S.image(S.Rng(103), 256),
                           fm=S.field_map(S.Rng(104), 8, 8, 4, 150.0), nc=2,
                           smap=S.coil_maps(S.Rng(105), 8, 8, 4, 2))
    # 2-D SENSE<TimeSegmentation<Gnufft>>, 32x32, L=4, 2 coils, +-100 Hz, 8 ms
    kx, ky, t = S.spiral(32, 4, 512, 8e-3)
    cases["tssense2d"] = dict(nx=32, ny=32, nz=1, kx=kx, ky=ky, kz=np.zeros_like(kx), t=t, L=4, nc=2,
                              fm=S.field_map(S.Rng(106), 32, 32, 1, 100.0),
                              smap=S.coil_maps(S.Rng(107), 32, 32, 1, 2), x=S.image(S.Rng(108), 1024))
    # 3-D pcSenseTimeSeg, 16x16x4, 2 shots, 2 coils, L=3
    kxs, kys, kzs, ts = [], [], [], []
    for s in range(2):
        a, b, c, d = S.stack_of_spirals(16, 4, 2, 128, 4e-3, which=[s])
        kxs.append(a); kys.append(b); kzs.append(c); ts.append(d)
    cases["pcsense3d"] = dict(nx=16, ny=16, nz=4, kx=np.concatenate(kxs), ky=np.concatenate(kys),
                              kz=np.concatenate(kzs), t=np.concatenate(ts), L=3, nc=2,
                              fm=S.field_map(S.Rng(109), 16, 16, 4, 200.0),
                              smap=S.coil_maps(S.Rng(110), 16, 16, 4, 2),
                              pmap=S.shot_phase_maps(S.Rng(111), 16, 16, 4, 2), x=S.image(S.Rng(112), 1024))
    # 3-D pcSENSE over Gdft, 8x8x4, 2 shots x 256 samples, 2 coils, +-150 Hz
    kxs, kys, kzs, ts = [], [], [], []
    for s in range(2):
        a, b, c, d = S.stack_of_spirals(8, 4, 2, 64, 20e-3, which=[s])
        kxs.append(a); kys.append(b); kzs.append(c); ts.append(d)
    cases["pcsense_gdft3d"] = dict(nx=8, ny=8, nz=4, kx=np.concatenate(kxs), ky=np.concatenate(kys),
                                   kz=np.concatenate(kzs), t=np.concatenate(ts), nc=2,
                                   fm=S.field_map(S.Rng(113), 8, 8, 4, 150.0),
                                   smap=S.coil_maps(S.Rng(114), 8, 8, 4, 2),
                                   pmap=S.shot_phase_maps(S.Rng(115), 8, 8, 4, 2), x=S.image(S.Rng(116), 256))
    # 3-D SENSE<GdftR2>, 8x8x4 image, 512 samples, +-150 Hz, 2 coils
    c = dict(cases["gdft3d"])
    c["x"] = S.image(S.Rng(117), 256)
    cases["gdftr2_3d"] = c
    # 2-D PCG: SENSE<TimeSegmentation<Gnufft>> + QuadPenalty, 5 iterations
    c = dict(cases["tssense2d"])
    c["beta"] = 1e-3
    c["niter"] = 5
    cases["pcg2d"] = c
    # 2-D PCG with TV
    c = dict(cases["tssense2d"])
    c["beta"] = 1e-2
    c["delta"] = 0.5
    c["niter"] = 5
    cases["pcgtv2d"] = c
    return cases


def build_op(name, c, prec):
    M = c["kx"].size
    n = c["nx"] * c["ny"] * c["nz"]
    if name.startswith("nufft"):
        return O.gnufft(prec, M, c["nx"], c["ny"], c["nz"], c["kx"], c["ky"], c["kz"])
    if name == "gdft3d":
        ix, iy, iz = S.image_coords(c["nx"], c["ny"], c["nz"])
        G = O.gdft(prec, c["kx"], c["ky"], c["kz"], ix, iy, iz, c["fm"], c["t"])
        return O.sense(G, c["smap"], M, n, c["nc"])
    if name == "gdftr2_3d":
        ix, iy, iz = S.image_coords(c["nx"], c["ny"], c["nz"])
        G = O.gdftr2(prec, c["kx"], c["ky"], c["kz"], ix, iy, iz, c["fm"], c["t"], c["nx"], c["ny"], c["nz"])
        return O.sense(G, c["smap"], M, n, c["nc"])
    if name == "pcsense3d":
        return O.pcsense_timeseg(prec, c["kx"], c["ky"], c["kz"], c["nx"], c["ny"], c["nz"], c["nc"], c["t"], c["L"],
                                 c["smap"], c["fm"], c["pmap"])
    if name == "pcsense_gdft3d":
        return O.pcsense(prec, c["kx"], c["ky"], c["kz"], c["nx"], c["ny"], c["nz"], c["nc"], c["t"], c["smap"],
                         c["fm"], c["pmap"])
    G = O.gnufft(prec, M, c["nx"], c["ny"], c["nz"], c["kx"], c["ky"], c["kz"])
    A = O.timeseg(G, c["fm"], c["t"], M, n, c["L"])
    return O.sense(A, c["smap"], M, n, c["nc"])


def compute(name, c, prec):
    """Outputs of one case at one precision with the current oracle backend."""
    op = build_op(name, c, prec)
    out = {}
    x = c["x"].astype(np.complex64 if prec == 0 else np.complex128)
    if name.startswith("pcg"):
        # data from the FP64 forward, cast to complex64 (as the bench forms it)
        op64 = build_op(name, c, 2)
        y = op64.forward(c["x"].astype(np.complex128)).astype(np.complex64)
        pen = "tv" if "delta" in c else "quad"
        xr, it = op.pcg(y, pen, c["nx"], c["ny"], c["nz"], c["beta"], c.get("delta", 1.0), 3, c["niter"])
        out["y"] = y
        out["x_pcg"] = xr
        out["iters"] = np.array(it)
        return out
    y = op.forward(x)
    out["y"] = y
    out["x_adj"] = op.adjoint(y)
    return out


def main(only=None):
    """Write every fixture, or only the named ones."""
    O.build(ref=True)
    O.use_reference(True)
    for name, c in small_cases().items():
        if only and name not in only:
            continue
        rec = {k: (np.asarray(v) if not np.isscalar(v) else np.array(v)) for k, v in c.items()}
        for prec, tag in ((0, "f32"), (2, "f64")):
            for k, v in compute(name, c, prec).items():
                rec[f"{k}_{tag}"] = v
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **rec)
        print("wrote", name)
    O.use_reference(False)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
