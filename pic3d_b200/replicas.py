"""Whole-job numbers for N independent replicas, one process per GPU.

The reference's only parallelism is MPI domain decomposition; this path
runs one domain per GPU with no exchange between GPUs, so N ranks are N
independent replicas.  The job's time is the slowest rank's device time and
its work is the sum of every rank's particle-steps.
"""
from __future__ import annotations


def combine(ms_local: float, particles_local: float, steps: int, dist=None, device=None):
    """(max ms over ranks, total particles, particle-steps/s of the job)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        ms, total = float(ms_local), float(particles_local)
    else:
        import torch
        t = torch.tensor([float(ms_local)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        n = torch.tensor([float(particles_local)], dtype=torch.float64, device=device)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
        ms, total = float(t.item()), float(n.item())
    return ms, total, total * steps / (ms / 1e3)
