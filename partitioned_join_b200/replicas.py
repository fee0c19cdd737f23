"""Multi-GPU runs of the join: independent replicas, one process per GPU.

The join does not exchange data between GPUs (the reference is a one-GPU
program and its partitions never leave the device), so N GPUs run N
replicas, each joining its own seeded inputs: weak scaling with no
data-path collective.  The only collectives are a barrier around the timed
region and the max over ranks of the timed duration, so the whole-job
throughput is (units every rank processed) / (slowest rank's time).
"""
from __future__ import annotations

import os
from typing import Tuple

import torch
import torch.distributed as dist


def world_from_env() -> Tuple[int, int, int]:
    """(rank, world_size, local_rank) as torchrun exports them; (0, 1, 0) alone."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(seed: int, rank: int) -> int:
    """Every replica joins different inputs of the same shape."""
    return seed + 1000003 * rank


def active() -> bool:
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def barrier() -> None:
    if active():
        dist.barrier()


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks (the slowest rank's time)."""
    if not active():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: int, device=None) -> int:
    """Total units processed by all ranks."""
    if not active():
        return int(value)
    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def whole_job_rate(units_all_ranks: int, max_ms: float) -> float:
    """Whole-job throughput: units of every rank per second of the slowest rank."""
    return units_all_ranks / (max_ms / 1e3) if max_ms > 0 else 0.0
