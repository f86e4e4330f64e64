"""Replica runs on several GPUs of one node: one process per GPU under torch.distributed.

The coupled epoch does not shard usefully (every substep would need a halo exchange, and one GPU
runs an epoch in milliseconds), so ranks run independent instances (replica seeds, or their share of
a campaign's instances) with no collective on the data path; only the timing is reduced, as the
maximum over ranks of each rank's device-timed region.
"""
from __future__ import annotations

import os


def dist_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment (torch.distributed.run)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} for world size {world}")
    return rank, world, local


def rank_share(items, rank: int, world: int) -> list:
    """This rank's share of a list of independent instances: every world-th item from `rank`."""
    return [x for i, x in enumerate(items) if i % world == rank]


def replica_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s replica of a seeded workload."""
    return int(seed) + int(rank)


def _reduce(value: float, op_name: str, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over the ranks of the default process group (the value itself without
    one). `device` must be the rank's CUDA device under NCCL; CPU under gloo."""
    return _reduce(value, "MAX", device)


def sum_over_ranks(value: float, device=None) -> float:
    """Sum of `value` over the ranks of the default process group (the value itself without one)."""
    return _reduce(value, "SUM", device)
