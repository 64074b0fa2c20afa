"""Replica plumbing for ``bench.py --gpus N`` (one process per GPU).

The timestep does not shard in this build: every rank advances its own
replica of the whole grid, and the ranks talk only to line up the timed
region (a barrier) and to take the slowest rank's time (a MAX all-reduce).
There is no data-path collective.  The process group uses NCCL on the GPUs
and gloo on CPU (the tests run two gloo ranks).
"""
from __future__ import annotations

import datetime
import os


def env():
    """(world size, rank, local rank) from the torchrun environment."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init(ws: int, backend: str = "nccl", timeout_s: float = 300.0) -> None:
    """Join the process group when there is more than one rank.  A short
    timeout makes a rank whose peers never arrive fail with an error instead
    of waiting for good."""
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def barrier(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v: float, ws: int, device: str = "cuda") -> float:
    """The largest value over the ranks (every rank gets it)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(ws: int, units_per_rank: float, max_seconds: float) -> float:
    """Units per second of the whole job: every rank processed the same
    units, and the job took as long as its slowest rank."""
    return ws * units_per_rank / max_seconds


def finish(ws: int) -> None:
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
