"""Multi-GPU layout: one reconstruction replica per GPU.

The path does not shard a single reconstruction (no collective sits inside
an operator or the solver); independent images run on separate GPUs, as
PowerGrid's MPI driver distributes them (MPI/PowerGridSenseMPI.cpp:197-250):
tasks enumerated slice-major with the repetition fastest (:206-219), dealt
round-robin over the ranks (:223-231), GPU = rank % GPUs (:236-241), images
gathered at rank 0.  One process per GPU under torchrun; the timing of a
multi-GPU run is the maximum over ranks.  torch.distributed carries the
plumbing: NCCL on GPUs, gloo on CPU (the tests).
"""
from __future__ import annotations

import os
from typing import Dict, List, Sequence, Tuple

__all__ = ["rank_layout", "task_list", "tasks_for_rank", "device_for_rank", "max_over_ranks", "job_rate",
           "gather_images"]


def rank_layout() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment (1, 0, 0 alone)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def task_list(n_slice: int, n_phase: int = 1, n_echo: int = 1, n_avg: int = 1,
              n_rep: int = 1) -> List[Tuple[int, int, int, int, int]]:
    """(slice, phase, echo, average, repetition) per task, in the reference's order."""
    return [(s, p, e, a, r) for s in range(n_slice) for p in range(n_phase) for e in range(n_echo)
            for a in range(n_avg) for r in range(n_rep)]


def tasks_for_rank(n_tasks: int, world_size: int, rank: int) -> List[int]:
    """Task indices of one rank: task t goes to rank t mod world_size."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} outside a world of {world_size}")
    return list(range(rank, n_tasks, world_size))


def device_for_rank(rank: int, n_gpus: int) -> int:
    if n_gpus < 1:
        raise ValueError("no GPUs")
    return rank % n_gpus


def max_over_ranks(x: float, device=None) -> float:
    """The largest x over the process group (x itself without one)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, seconds_max: float, world_size: int) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    if seconds_max <= 0:
        raise ValueError("non-positive time")
    return world_size * units_per_rank / seconds_max


def gather_images(local: Dict[int, object], world_size: int) -> Dict[int, object]:
    """Rank 0 receives every rank's {task: image}; the other ranks get {}."""
    import torch.distributed as dist
    if world_size == 1 or not dist.is_initialized():
        return dict(local)
    rank = dist.get_rank()
    parts: Sequence = [None] * world_size if rank == 0 else None
    dist.gather_object(local, parts, dst=0)
    if rank != 0:
        return {}
    out: Dict[int, object] = {}
    for p in parts:
        out.update(p)
    return out
