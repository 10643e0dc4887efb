"""Multi-GPU plumbing: one process per GPU, launched by torchrun.

The path shards only across scenes.  A single scene does not shard (its
Poisson solve couples the whole grid), so N GPUs run N replicas of it; a batch
of independent scenes (the 64-scene mix) is split by whole scenes, each rank
running its share through the batch entry point.  No data crosses ranks: the
only collectives are the barrier around the timed region and the maximum of
the ranks' device times.  Everything here runs on the gloo backend on CPU as
well, which is how the tests cover it.
"""
from __future__ import annotations

import os
from datetime import timedelta
from typing import Sequence

import torch
import torch.distributed as dist


def env_ranks() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment (1, 0, 0 alone)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(world: int, rank: int, backend: str, timeout_s: float = 120.0, device=None) -> None:
    """Process group with a short timeout, so that ranks waiting for a rank
    that left end with an error instead of hanging."""
    if world <= 1 or dist.is_initialized():
        return
    kw = {"timeout": timedelta(seconds=timeout_s)}
    if backend == "nccl" and device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)


def scene_cost(grid_edge: int, particles: int) -> float:
    """Predicted device time of one scene step, in arbitrary units: the grid
    stages scale with the cells, the hash and near field with the particles
    (the two terms are of equal weight for a 128^3 grid with 1M particles)."""
    return float(grid_edge) ** 3 + 2.0 * float(particles)


def partition_scenes(costs: Sequence[float], world: int) -> list[list[int]]:
    """Whole scenes to ranks, longest first onto the least-loaded rank (LPT).
    Deterministic: every rank computes the same partition.  Returns, per
    rank, its scene indices in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, device: torch.device | str = "cpu") -> float:
    """The maximum of a per-rank scalar (a device time) over all ranks."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device: torch.device | str = "cpu") -> float:
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier() -> None:
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def finish() -> None:
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
