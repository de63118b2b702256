"""Replica layout of the multi-GPU benchmark: one process per GPU, each an
independent copy of the single-GPU workload (the eigensolver inner loop is
run on one GPU per cell; there is no data-path collective).  The only
exchanges are the timing barrier and the max-over-ranks reduction of the
per-rank times, so the whole-job rate is replicas x bands x iterations over
the slowest rank's time.
"""
from __future__ import annotations

import datetime
import os


def rank_info(env=None):
    """(rank, world size, local rank) from the torchrun environment."""
    env = os.environ if env is None else env
    return int(env.get("RANK", "0")), int(env.get("WORLD_SIZE", "1")), int(env.get("LOCAL_RANK", "0"))


def init(world: int, backend: str = "nccl", timeout_s: int = 120):
    """Process group for world > 1 (short timeout: a missing rank ends the
    next collective with an error instead of a hang); None for one process."""
    if world <= 1:
        return None
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(value: float, dist, device=None) -> float:
    """The slowest rank's value (every rank takes part, in the same order)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(per_rank_units: float, world: int, max_seconds: float) -> float:
    """Units processed by all ranks over the slowest rank's time."""
    return world * per_rank_units / max_seconds
