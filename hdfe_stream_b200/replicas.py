"""Several GPUs, one process each: every rank fits its own panel.

A fit has no data-path exchange -- its rows, cells, S and solve live on one
GPU -- so N ranks are N independent replicas (weak scaling): the only
collectives are the timing barrier and the max over ranks of the device
time, and the whole job's rate is the units all ranks processed over that
time.  These helpers are what `bench.py --gpus N` uses under torchrun; the
backend is NCCL on GPUs and gloo for the CPU tests of the same logic.
"""

from __future__ import annotations

import datetime


def init(world: int, backend: str = "nccl", device=None, timeout_s: float = 600.0):
    """The process group for `world` > 1 ranks (env:// rendezvous), or None."""
    if world <= 1:
        return None
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def max_over_ranks(value: float, dist, device="cpu") -> float:
    """The largest of the ranks' values (the job's time is its slowest rank's)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, ms: float, world: int) -> float:
    """Units per second for the whole job: every rank's units over the
    max-over-ranks time in milliseconds."""
    return world * float(units_per_rank) / (float(ms) / 1e3)


def rank_seed(rank: int, base: int = 0) -> int:
    """Each rank's panel seed: replicas fit different data."""
    return base + int(rank)
