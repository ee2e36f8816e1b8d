"""Replica-parallel bookkeeping for multi-GPU runs.

The path has no exchange step (the reference is single-GPU; SRC/setup.F90:45
fixes myrank = 0), so N GPUs run N independent lattices.  The only
inter-process traffic is timing: every rank reports its device time and its
lattice updates; the job throughput is all updates over the slowest rank's
time (max over ranks).
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def job_throughput(local_updates: float, local_seconds: float, device=None) -> tuple[float, float, float]:
    """Returns (total_updates, max_seconds, updates_per_second) over all ranks.
    Works with any initialised process group (nccl on GPUs, gloo on CPU);
    without one it returns the local figures."""
    if not (dist.is_available() and dist.is_initialized()):
        return local_updates, local_seconds, local_updates / local_seconds
    dev = device if device is not None else ("cuda" if dist.get_backend() == "nccl" else "cpu")
    t = torch.tensor([local_seconds], dtype=torch.float64, device=dev)
    u = torch.tensor([local_updates], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(u.item()), float(t.item()), float(u.item()) / float(t.item())
