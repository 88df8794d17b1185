"""Replica launch helpers shared by bench.py and the multi-process tests.

Rows of a batched FFT are independent, so N GPUs run N replicas of the
workload (one process per GPU, weak scaling) with no data-path collective.
The only collectives are a barrier around the timed region and a MAX
reduction of each rank's device-measured time, so that a step's time is the
slowest replica's.
"""
from __future__ import annotations

import os


def rank_env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """MAX of `value` over the process group (the value itself without one).
    `device` is where the reduction tensor lives: the rank's GPU under NCCL,
    the CPU under gloo."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reports(rank: int) -> bool:
    """Only rank 0 prints the result line."""
    return rank == 0
