"""Replica-parallel runs: one process per GPU, each stepping its own copy of
the workload (cases are independent; the time step has no exchange between
them).  The job's time is the slowest rank's, its work the sum over ranks.

Used by bench.py under torchrun (NCCL, device tensors) and tested with gloo
ranks on CPU.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def world() -> tuple[int, int]:
    """(rank, world size) of the current process group, (0, 1) without one."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def max_over_ranks(x: float, device: torch.device | None = None) -> float:
    """The largest value of x over all ranks (x itself without a group)."""
    r, n = world()
    if n == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device: torch.device | None = None) -> float:
    r, n = world()
    if n == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_this_rank: float, ms_this_rank: float,
             device: torch.device | None = None) -> tuple[float, float]:
    """(whole-job units per second, job milliseconds): every rank's units over
    the slowest rank's time."""
    ms = max_over_ranks(ms_this_rank, device)
    units = sum_over_ranks(units_this_rank, device)
    return units / (ms / 1e3), ms
