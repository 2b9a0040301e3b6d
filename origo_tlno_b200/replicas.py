"""Multi-GPU replicas: one process per GPU, each building the J/K of its own
copy of the workload (a J/K build of one molecule is not sharded; the work
of different molecules or replicas needs no exchange).  The only collective
is the timing reduction: the step time is the maximum over ranks, and the
whole-job throughput is the sum of the units all ranks processed divided by
that time.
"""
from __future__ import annotations

import datetime
import os


def world():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0):
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(values, device=None):
    """Elementwise maximum of a list of floats over all ranks (identity for
    one process)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def throughput(units_per_rank: float, seconds_max: float, world_size: int) -> float:
    """Whole-job units per second: every rank processes units_per_rank in at
    most seconds_max."""
    return world_size * units_per_rank / seconds_max
