"""Replica dispatch for N GPUs (one process per GPU, torch.distributed for the plumbing).

A stereo pair does not shard: its vertical and diagonal SGM paths need whole columns, so
splitting one pair across GPUs would need a transpose exchange for sub-GB volumes.  Multi-GPU
work is therefore independent replicas: rank r processes pairs r, r+N, r+2N, ... and nothing is
exchanged on the data path.  The only collectives are the host-side barrier and the max of the
per-rank device times used for whole-job throughput.
"""
from __future__ import annotations

from typing import Callable, Sequence


def assign(n_items: int, rank: int, world: int) -> list[int]:
    """Indices of the items rank `rank` of `world` processes (round robin)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("invalid rank/world")
    return list(range(rank, n_items, world))


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank scalar over all ranks (the job's wall time is set by the slowest)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def run_replica(items: Sequence, process: Callable, rank: int, world: int) -> dict:
    """Process this rank's share of `items`; returns {index: result}."""
    return {i: process(items[i]) for i in assign(len(items), rank, world)}


def throughput(units_per_rank: Sequence[float], times_per_rank: Sequence[float]) -> float:
    """Whole-job throughput: all units processed by all ranks over the slowest rank's time."""
    return float(sum(units_per_rank)) / max(times_per_rank)
