"""The header-only C++ operator API, compiled here with g++ and run on the GPU."""
import os
import subprocess

import numpy as np
import pytest

from conftest import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "recon_api.cpp")
LIBDIR = os.path.join(ROOT, "powergrid_b200", "lib")


def _build(outdir):
    exe = os.path.join(outdir, "recon_api")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L" + LIBDIR, "-lpowergrid_b200", "-Wl,-rpath," + LIBDIR], check=True)
    return exe


def test_cpp_api_compiles(tmp_path):
    from powergrid_b200 import build as B
    B.build()
    assert os.path.exists(_build(str(tmp_path)))


@pytest.mark.gpu
def test_cpp_api_matches_reference_fixture(pg, tmp_path):
    d = np.load(os.path.join(ROOT, "tests", "golden", "pcg2d.npz"))
    c = {k: d[k] for k in d.files}
    nx, ny, nz, L, nc, niter = (int(c[k]) for k in ("nx", "ny", "nz", "L", "nc", "niter"))
    M = c["kx"].size
    out = str(tmp_path)
    with open(os.path.join(out, "meta.txt"), "w") as f:
        f.write(f"{nx} {ny} {nz} {M} {L} {nc} {niter} {float(c['beta'])}\n")
    for k, dt in (("kx", np.float32), ("ky", np.float32), ("kz", np.float32), ("t", np.float32),
                  ("fm", np.float32), ("smap", np.complex64), ("x", np.complex64)):
        np.ascontiguousarray(c[k], dtype=dt).tofile(os.path.join(out, k + ".bin"))
    np.ascontiguousarray(c["y_f32"], dtype=np.complex64).tofile(os.path.join(out, "data.bin"))
    exe = _build(out)
    subprocess.run([exe, out], check=True)
    y = np.fromfile(os.path.join(out, "y_out.bin"), np.complex64)
    img = np.fromfile(os.path.join(out, "img_out.bin"), np.complex64)
    t = np.load(os.path.join(ROOT, "tests", "golden", "tssense2d.npz"))
    assert rel_l2(y, t["y_f32"]) <= 1e-5          # same geometry and image as the tssense2d fixture
    assert rel_l2(img, c["x_pcg_f32"]) <= 1e-4    # reconSolve, 5 iterations
    # the C++ helpers return what the Python API does (same library calls)
    dcf = np.fromfile(os.path.join(out, "dcf_out.bin"), np.float32)
    sos = np.fromfile(os.path.join(out, "sos_out.bin"), np.float32)
    assert np.array_equal(dcf, pg.calc3DDensityCompensation(c["kx"], c["ky"], c["kz"], nx, nz))
    G = pg.Gnufft(M, 2.0, nx, ny, nz, c["kx"], c["ky"], c["kz"])
    coil = pg.gridCoilImages(G, dcf, c["y_f32"], nc)
    assert rel_l2(sos, pg.calcSumOfSquaresImage(coil, nc)) <= 1e-6
    rt = np.fromfile(os.path.join(out, "interp_out.bin"), np.complex64)
    ysub = y[:M]
    assert rt.size == M and rel_l2(rt, G.forwardSpatialInterp(G.adjointSpatialInterp(ysub))) <= 1e-6
    # LRobj over two copies of the SENSE operator with an identity basis: each
    # repetition's data is that operator's output; the solve runs the same
    # library path as the Python API
    ylr = np.fromfile(os.path.join(out, "ylr_out.bin"), np.complex64)
    assert np.array_equal(ylr, np.concatenate([y, y]))
    xlr = np.fromfile(os.path.join(out, "xlr_out.bin"), np.complex64)
    A = pg.TimeSegmentation(G, c["fm"], c["t"], M, nx * ny * nz, L, 1, 1)
    S = pg.SENSE(A, c["smap"], M, nx * ny * nz, nc)
    v = np.eye(2, dtype=np.complex64)
    Alr = pg.LRobj(nx * ny * nz, M * nc, 2, 2, v, [S, S])
    xp, _ = pg.solve_pwls_pcg(None, Alr, None, np.concatenate([c["y_f32"]] * 2),
                              pg.R_lowRank(pg.QuadPenalty(nx, ny, nz, float(c["beta"])), 2, 2, v), 3)
    assert rel_l2(xlr, xp) <= 1e-6
    # NIfTI magnitude/phase of the solved image; the gathered acquisitions
    # reproduce the data and trajectory they were cut from (M even here)
    from powergrid_b200 import ingest
    ingest.writeNiftiMagPhsImage(os.path.join(out, "py"), img, nx, ny, nz)
    for part in ("_mag.nii", "_phs.nii"):
        a = np.fromfile(os.path.join(out, "img" + part), np.uint8)
        assert np.array_equal(a, np.fromfile(os.path.join(out, "py" + part), np.uint8))
    gd = np.fromfile(os.path.join(out, "gather_data.bin"), np.complex64)
    assert np.array_equal(gd, c["y_f32"].astype(np.complex64))
    assert np.array_equal(np.fromfile(os.path.join(out, "gather_kx.bin"), np.float32), c["kx"].astype(np.float32))
    # pg::Server: the image as a request and as the driver's loop over the index equals reconSolve's
    for name in ("served_req.bin", "served_acq.bin"):
        e = rel_l2(np.fromfile(os.path.join(out, name), np.complex64), img)
        print(f"{name}: vs reconSolve {e:.2e}")
        assert e <= 1e-5
