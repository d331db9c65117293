"""The multi-GPU plumbing as two gloo ranks on CPU: the reference MPI driver's
task layout (MPI/PowerGridSenseMPI.cpp:206-241), max-over-ranks timing, and
the gather of every rank's images at rank 0, each rank reconstructing its
share of the tasks (the oracle stands in for a GPU here)."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from powergrid_b200 import replicas as R


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _task_image(task):
    """The adjoint of one task's seeded data through the oracle's Gnufft (16x16)."""
    import oracle as O
    from powergrid_b200 import synthetic as S
    n = 16
    kx, ky, _ = S.spiral(n, 2, 128, 4e-3)
    G = O.gnufft(0, kx.size, n, n, 1, kx, ky, np.zeros_like(kx))
    return G.adjoint(S.image(S.Rng(500 + task), kx.size))


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        layout = R.rank_layout()
        tasks = R.task_list(3, 1, 1, 1, 2)
        mine = R.tasks_for_rank(len(tasks), ws, rank)
        images = {t: _task_image(t) for t in mine}
        gathered = R.gather_images(images, ws)
        tmax = R.max_over_ranks(1.0 + rank)
        rate = R.job_rate(20 * len(mine), tmax, ws)
        q.put((rank, layout, mine, gathered, tmax, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = {}
        for _ in range(2):
            rank, *rest = q.get(timeout=120)
            res[rank] = rest
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert res[0][0] == (2, 0, 0) and res[1][0] == (2, 1, 1)
    assert res[0][1] == [0, 2, 4] and res[1][1] == [1, 3, 5]          # round-robin over 6 tasks
    gathered = res[0][2]
    assert sorted(gathered) == list(range(6)) and res[1][2] == {}
    for t, img in gathered.items():
        assert np.array_equal(img, _task_image(t))                    # same as one process computing it
    assert res[0][3] == res[1][3] == 2.0                              # the slower rank's time
    assert res[0][4] == res[1][4] == 2 * 20 * 3 / 2.0


def test_layout_rules():
    tasks = R.task_list(2, 1, 2, 1, 3)
    assert len(tasks) == 12 and tasks[:4] == [(0, 0, 0, 0, 0), (0, 0, 0, 0, 1), (0, 0, 0, 0, 2), (0, 0, 1, 0, 0)]
    assert R.tasks_for_rank(5, 3, 2) == [2] and R.tasks_for_rank(2, 4, 3) == []
    assert [R.device_for_rank(r, 8) for r in (0, 7, 8, 13)] == [0, 7, 0, 5]
    assert R.max_over_ranks(3.5) == 3.5                               # no process group
    with pytest.raises(ValueError):
        R.tasks_for_rank(4, 2, 2)
    with pytest.raises(ValueError):
        R.job_rate(1.0, 0.0, 1)
