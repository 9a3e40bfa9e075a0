"""Runs on several GPUs of one node.

The density update has no exchange step between independent grids, so N GPUs
run N replicas: every rank advances its own grid (its own seed), nothing
crosses NVLink on the data path, and a job's time is the slowest rank's
(one all-reduce of a scalar after the timed region).  Works with any
torch.distributed backend: NCCL on the GPUs, gloo on CPU for the tests.
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass
class RankInfo:
    rank: int
    world: int
    local: int


def rank_info() -> RankInfo:
    """RANK / WORLD_SIZE / LOCAL_RANK as torchrun sets them (1 rank without)."""
    return RankInfo(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x: float, device: str = "cuda") -> float:
    """The largest value of x over the ranks (x itself for one rank)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def job_throughput(units_per_rank: float, world: int, seconds: float) -> float:
    """Whole-job throughput: the units every rank processed over the slowest
    rank's time."""
    return world * units_per_rank / seconds
