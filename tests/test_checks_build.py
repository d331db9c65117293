"""The PG_CHECKS build (libpowergrid_b200_checks.so): the gridding kernels with
their device-side index checks compiled in.  A check that fails records
(site, value) in a device word and skips the access instead of trapping;
pg_checks_read returns the first record.

The GPU test runs the checks library in a subprocess (the package loads one
library per process, chosen by PG_LIBRARY) over the 2-D fused and tiled
gridding paths (several tiles and coils per item), the 3-D path and a PCG
solve, and requires every check to pass with results equal to the oracle's
within the operator tolerance.  No test makes a check fail on the GPU: the
checks guard indices derived from the binning, which the host validates, so
a failing check would need a corrupted binning.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, os, sys
sys.path.insert(0, os.path.join(ROOT, "oracle")); sys.path.insert(0, ROOT)
import ctypes as C
import numpy as np
import oracle as O
import powergrid_b200 as pg
from powergrid_b200 import _lib, synthetic as S

assert _lib.LIB_PATH.endswith("libpowergrid_b200_checks.so"), _lib.LIB_PATH
pg.init(0)

def rel(a, b):
    return float(np.linalg.norm(a.astype(np.complex128) - b) / np.linalg.norm(b.astype(np.complex128)))

def read():
    rec, en = C.c_uint64(), C.c_int()
    _lib.check(_lib.load().pg_checks_read(C.byref(rec), C.byref(en)))
    return int(rec.value), int(en.value)

out = {"cases": []}
n, nc, L = 32, 3, 4
kx, ky, t = S.spiral(n, 4, 768, 8e-3)
kz = np.zeros_like(kx)
fm = S.field_map(S.Rng(401), n, n, 1, 100.0)
sm = S.coil_maps(S.Rng(402), n, n, 1, nc)
x = S.image(S.Rng(403), n * n)
M = kx.size
So = O.sense(O.timeseg(O.gnufft(0, M, n, n, 1, kx, ky, kz), fm, t, M, n * n, L), sm, M, n * n, nc)
yo = So.forward(x)
xo = So.adjoint(yo)
for tile, cc in ((16, 2), (32, 1), (16, 4)):
    os.environ.update(PG_AUTOTUNE="0", PG_TILE2D=str(tile), PG_SPREAD_CC=str(cc), PG_GATHER_CC=str(cc))
    G = pg.Gnufft(M, 2.0, n, n, 1, kx, ky, kz)
    A = pg.TimeSegmentation(G, fm, t, M, n * n, L, 1, 1)
    Sg = pg.SENSE(A, sm, M, n * n, nc)
    ef, ea = rel(Sg * x, yo), rel(Sg / yo, xo)
    rec, en = read()
    out["cases"].append({"case": f"2-D TS-SENSE tile {tile}, {cc} coils per item", "fwd": ef, "adj": ea,
                         "record": rec, "enabled": en})
xs = pg.reconSolve(yo, Sg, pg.QuadPenalty(n, n, 1, 1e-3), niter=3)
xr, _ = So.pcg(yo, "quad", n, n, 1, 1e-3, niter=3)
rec, en = read()
out["cases"].append({"case": "2-D PCG, 3 iterations", "pcg": rel(xs, xr), "record": rec, "enabled": en})
n3, nz = 16, 8
a, b, c, t3 = S.stack_of_spirals(n3, nz, 4, 512, 6e-3)
G3 = pg.Gnufft(a.size, 2.0, n3, n3, nz, a, b, c)
G3o = O.gnufft(0, a.size, n3, n3, nz, a, b, c)
x3 = S.image(S.Rng(404), n3 * n3 * nz)
y3 = G3o.forward(x3)
ef, ea = rel(G3 * x3, y3), rel(G3 / y3, G3o.adjoint(y3))
rec, en = read()
out["cases"].append({"case": "3-D Gnufft 16x16x8", "fwd": ef, "adj": ea, "record": rec, "enabled": en})
print("CHECKS " + json.dumps(out))
"""


@pytest.mark.gpu
def test_checks_build_runs_clean():
    lib = os.path.join(ROOT, "powergrid_b200", "lib", "libpowergrid_b200_checks.so")
    if not os.path.exists(lib):
        from powergrid_b200 import build as B
        B.build(checks=True)
    env = dict(os.environ, PG_LIBRARY="checks")
    r = subprocess.run([sys.executable, "-c", "ROOT = " + repr(ROOT) + "\n" + SCRIPT], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("CHECKS ")][-1]
    res = json.loads(line[len("CHECKS "):])
    for case in res["cases"]:
        print(case)
        assert case["enabled"] == 1 and case["record"] == 0, case
        for k in ("fwd", "adj"):
            if k in case:
                assert case[k] <= 1e-5, case
        if "pcg" in case:
            assert case["pcg"] <= 1e-4, case


def test_both_libraries_export_the_checks_reader():
    """Both libraries export pg_checks_read (the product answers enabled = 0);
    loading needs no GPU."""
    import ctypes as C
    for name in ("libpowergrid_b200.so", "libpowergrid_b200_checks.so"):
        path = os.path.join(ROOT, "powergrid_b200", "lib", name)
        if not os.path.exists(path):
            pytest.skip(f"{name} not built")
        lib = C.CDLL(path)
        assert hasattr(lib, "pg_checks_read")
