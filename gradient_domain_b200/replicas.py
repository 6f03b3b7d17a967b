"""Replica parallelism across the GPUs of one node.

Instances, channels and requests of this path are independent, so several
GPUs run as replicas: one process per GPU, each with its own instances and no
collective on the data path.  Only the start barrier and the max-over-ranks
step time cross processes (NCCL on GPUs; the same code runs on ``gloo`` for
the CPU tests).
"""

from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def rank_env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(world: int, backend: str = "nccl", timeout_s: float = 120.0) -> None:
    """Join the process group when there is more than one rank; a short timeout
    turns a rank that never arrives into an error instead of a hang."""
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def finish(world: int) -> None:
    if world > 1 and dist.is_initialized():
        dist.destroy_process_group()


def barrier(world: int) -> None:
    if world > 1:
        dist.barrier()


def replica_seed(base: int, rank: int) -> int:
    """Each replica solves its own seeded instances (weak scaling)."""
    return base + rank


def max_over_ranks(value: float, world: int, device: torch.device | str = "cpu") -> float:
    """The slowest rank's time: the job's step time."""
    if world == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Whole-job throughput: every rank processed `units_per_rank` in `seconds`
    (the max over ranks)."""
    return units_per_rank * world / seconds


def split_evenly(items, rank: int, world: int):
    """Round-robin share of a fixed list (strong scaling of a request set)."""
    return list(items)[rank::world]
