"""Replica plumbing for multi-GPU runs: one process per GPU (torchrun), each
rank solving its own seeded copy of the workload. The solve path has no
exchange step, so there is no collective on the data path; the only
collectives are the barrier around the timed region and the max over ranks of
the device time."""
from __future__ import annotations

import datetime
import os


def rank_env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 600):
    """Process group for world_size > 1 (None otherwise)."""
    world, _, _ = rank_env()
    if world <= 1:
        return None
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank scalar (device time of the timed region)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: int, ms_max: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return world * units_per_rank / (ms_max / 1e3)


def shard(count: int, world: int, rank: int) -> range:
    """Contiguous share of `count` independent units (grids, requests) for a
    rank; shares differ by at most one unit and cover every unit once."""
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def replica_seed(seed: int, rank: int) -> int:
    """Seed of a rank's copy of the workload."""
    return seed + rank
