"""The allocation-free Gdft forward (pg_gdft_forward_noalloc).

Callers that own all device memory (their own pool, a fixed budget) or must
avoid cudaMalloc's implicit synchronisation cannot use an entry point that
allocates; this one keeps its scratch in a fixed device array.  The test
calls it through the C ABI twice in a row on caller-owned device buffers and
checks each result against the existing Gdft operator (pg_op_forward_device)
and against the oracle's restatement of the reference's float ftCpu, within
the operator tolerance.  During those calls the library's allocation hook is
armed to fail the next device allocation, so a call that allocated would
return PG_OUT_OF_MEMORY.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

OP_TOL = 1e-5


def _dev(a, torch, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.mark.gpu
def test_noalloc_gdft_matches_operator_twice(pg, oracle):
    import torch

    from powergrid_b200 import _lib
    from powergrid_b200 import synthetic as S
    from powergrid_b200._lib import P, check

    dev = torch.device("cuda", 0)
    kx, ky, kz, t = S.stack_of_spirals(16, 8, 1, 512, 25e-3)      # 4096 samples
    ix, iy, iz = S.image_coords(16, 16, 8)                          # 2048 voxels
    fm = S.field_map(S.Rng(21), 16, 16, 8, 150.0)
    nk, ni = kx.size, ix.size
    G = pg.Gdft(nk, ni, kx, ky, kz, ix, iy, iz, fm, t)
    L = _lib.load()
    R = oracle.gdft(0, kx, ky, kz, ix, iy, iz, fm, t)
    inputs = [_dev(v, torch, dev) for v in (kx, ky, kz, ix, iy, iz, fm, t)]
    stream = torch.cuda.current_stream()
    y = torch.empty(nk, dtype=torch.complex64, device=dev)
    try:
        for seed in (31, 32):                         # two calls in a row, different images
            img = S.image(S.Rng(seed), ni)
            x = _dev(img, torch, dev)
            y_op = G.forward(x, stream=stream)        # the existing entry point
            torch.cuda.synchronize()
            L.pg_debug_fail_allocation_after(1)       # any library allocation now fails
            check(L.pg_gdft_forward_noalloc(nk, ni, *[P(v.data_ptr()) for v in inputs], P(x.data_ptr()),
                                            P(y.data_ptr()), P(stream.cuda_stream)))
            L.pg_debug_fail_allocation_after(0)
            torch.cuda.synchronize()
            got, y_op = y.cpu().numpy(), y_op.cpu().numpy()
            e_op, e_or = rel_l2(got, y_op), rel_l2(got, R.forward(img))
            print(f"no-alloc Gdft: {e_op:.2e} vs the Gdft operator, {e_or:.2e} vs the oracle")
            assert e_op <= OP_TOL and e_or <= OP_TOL, (e_op, e_or)
    finally:
        L.pg_debug_fail_allocation_after(0)


@pytest.mark.gpu
def test_noalloc_gdft_rejects_oversized(pg):
    import torch

    from powergrid_b200 import _lib
    from powergrid_b200._lib import P, PGError, check

    dev = torch.device("cuda", 0)
    nk = (1 << 19) + 1
    buf = torch.zeros(nk, dtype=torch.float32, device=dev)
    xy = torch.zeros(2 * nk, dtype=torch.float32, device=dev)
    ptrs = [P(buf.data_ptr())] * 8
    with pytest.raises(PGError, match="INVALID_ARG"):
        check(_lib.load().pg_gdft_forward_noalloc(nk, 16, *ptrs, P(xy.data_ptr()), P(xy.data_ptr()), None))
    _ = C
