"""The one-cluster PCG steps of small problems (image and data of at most 4096
entries per slice, quadratic penalty; one cluster per slice of a stacked
solve): k_image_step_quad does the work of k_ngrad + k_ddir_quad and
k_data_step_quad that of k_daw + k_update, with cluster barriers where the
separate kernels have launch boundaries.  Their per-entry arithmetic is the
separate kernels'; only the FP64 sums are added in another fixed order.  A
solve through them must give the image and the iteration count of the
separate kernels (PG_IMAGE_STEP=0), for one solve and for the slices of a
served request solved as one stacked problem.  The switch is read once per
process, so each form runs in a subprocess; 3 iterations keep the comparison
below the point where CG amplifies the adjoint's float-atomic ordering.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import os, sys
sys.path.insert(0, ROOT)
import numpy as np
import powergrid_b200 as pg
from powergrid_b200 import synthetic as S
pg.init(0)
out = {}
p = S.config1()                                    # 64x64, one coil, 4096 samples
M, n = p.kx.size, p.nimg
G = pg.Gnufft(M, 2.0, p.nx, p.ny, 1, p.kx, p.ky, p.kz)
Sg = pg.SENSE(G, p.smap, M, n, 1)
y = (Sg * p.x_true).astype(np.complex64)
x, it = pg.solve_pwls_pcg(None, Sg, None, y, pg.QuadPenalty(p.nx, p.ny, 1, p.beta), 3)
out["cfg1"] = (x, it)
n2, nc, L = 32, 2, 4                               # 32x32 TS-SENSE, 2 coils: data 2 x 2048
kx, ky, t = S.spiral(n2, 4, 512, 8e-3)
kz = np.zeros_like(kx)
G2 = pg.Gnufft(kx.size, 2.0, n2, n2, 1, kx, ky, kz)
A2 = pg.TimeSegmentation(G2, S.field_map(S.Rng(501), n2, n2, 1, 100.0), t, kx.size, n2 * n2, L, 1, 1)
S2 = pg.SENSE(A2, S.coil_maps(S.Rng(502), n2, n2, 1, nc), kx.size, n2 * n2, nc)
y2 = (S2 * S.image(S.Rng(503), n2 * n2)).astype(np.complex64)
x2, it2 = pg.solve_pwls_pcg(None, S2, None, y2, pg.QuadPenalty(n2, n2, 1, 1e-3), 3)
out["ts32"] = (x2, it2)
# three slices served as one stacked solve (one cluster per slice): data 2 x 2048 per slice
from powergrid_b200.serve import ReconRequest, Server
ns = 3
fms = np.concatenate([S.field_map(S.Rng(510 + k), n2, n2, 1, 80.0) for k in range(ns)])
sms = np.concatenate([S.coil_maps(S.Rng(520 + k), n2, n2, 1, nc) for k in range(ns)])
ys = []
for k in range(ns):
    Ak = pg.TimeSegmentation(G2, fms[k * n2 * n2:(k + 1) * n2 * n2], t, kx.size, n2 * n2, L, 1, 1)
    Sk = pg.SENSE(Ak, sms[k * n2 * n2 * nc:(k + 1) * n2 * n2 * nc], kx.size, n2 * n2, nc)
    ys.append((Sk * S.image(S.Rng(530 + k), n2 * n2)).astype(np.complex64))
req = ReconRequest(n2, n2, 1, nc, L, 3, 1e-3, kx, ky, kz, t, fms, sms, np.concatenate(ys), ns)
srv = Server(hbm_budget_bytes=8 << 30, max_inflight=1)
img, st = srv.wait(srv.submit(req))
srv.close()
assert st["status"] == "PG_OK" and st["jobs"] == 1, st
out["served3"] = (img.ravel(), st["iters_done"] // ns)
np.savez(OUT, **{k + "_x": v[0] for k, v in out.items()}, **{k + "_it": np.array(v[1]) for k, v in out.items()})
"""


def _run(tmp_path, tag, env_extra):
    path = str(tmp_path / f"{tag}.npz")
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", f"ROOT = {ROOT!r}\nOUT = {path!r}\n" + SCRIPT], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(path)


@pytest.mark.gpu
def test_cluster_steps_match_separate_kernels(pg, tmp_path):
    fused = _run(tmp_path, "fused", {})
    sep = _run(tmp_path, "separate", {"PG_IMAGE_STEP": "0"})
    for case in ("cfg1", "ts32", "served3"):
        e = rel_l2(fused[case + "_x"], sep[case + "_x"])
        print(f"{case}: cluster steps vs separate kernels {e:.2e}, iterations {int(fused[case + '_it'])}")
        assert int(fused[case + "_it"]) == int(sep[case + "_it"]) == 3
        assert e <= 1e-5
