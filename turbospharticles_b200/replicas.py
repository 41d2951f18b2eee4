"""Replica plumbing for multi-GPU runs.

The IISPH step does not shard without the reference's MPI halo exchange (outside this
path), so N GPUs run N independent scenes ("replicas", weak scaling): one process per GPU,
launched by torchrun; `torch.distributed` is used only to line the ranks up (barrier) and to
take the maximum of the per-rank device times. No particle data crosses GPUs.
"""
from __future__ import annotations

import datetime
import os


def dist_env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, world_size: int, timeout_s: float = 120.0):
    """Process group for world_size > 1 (None otherwise); a short timeout makes ranks that wait
    for a rank that left fail with an error instead of waiting for ever."""
    if world_size <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(dist, device=None):
    if dist is None:
        return
    import torch
    if device is not None and device.type == "cuda":
        dist.all_reduce(torch.zeros(1, device=device))
    else:
        dist.barrier()


def max_over_ranks(dist, value: float, device=None) -> float:
    """Maximum of a per-rank scalar (the job's device time is the slowest rank's)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: int, world_size: int, max_ms: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return units_per_rank * world_size / (max_ms / 1e3)


def replica_seed(base_seed: int, rank: int) -> int:
    """Each replica scene gets its own jitter seed."""
    return int(base_seed) + 7919 * int(rank)
