"""Multi-GPU runs as replicas: one process per GPU, each running its own independent solve.

The solve does not shard in this build (no data-path collective), so N GPUs run N replicas of
the same workload. A rate over the whole job counts the units of every rank and divides by the
slowest rank's device time. That time is the maximum over ranks of each rank's CUDA-event time,
reduced with torch.distributed (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass(frozen=True)
class RankEnv:
    world: int
    rank: int
    local: int


def rank_env() -> RankEnv:
    """WORLD_SIZE / RANK / LOCAL_RANK as torch.distributed.run sets them (1 / 0 / 0 without it)."""
    return RankEnv(int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                   int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The largest x over all ranks (every rank must call it, in the same order)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, slowest_seconds: float) -> float:
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return units_per_rank * world / slowest_seconds
