"""Replica plumbing for one process per GPU (torch.distributed): the path does not shard, so
ranks evolve independent lattices (or tempering streams) and only scalars cross ranks.

job_rate(): whole-job throughput = units done by all ranks / the slowest rank's device time.
gather_streams(): every rank learns every stream's (Q, scale) for the tempering decisions,
which each rank then computes identically from a shared seed (tempering.swap_decisions).
"""
from __future__ import annotations


def reduce_max(x: float, dist=None, device: str = "cpu") -> float:
    if dist is None or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float, dist=None, device: str = "cpu") -> float:
    if dist is None or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units: float, ms: float, dist=None, device: str = "cpu") -> tuple[float, float]:
    """(units of all ranks per second over the slowest rank's time, that time in ms)."""
    total = reduce_sum(units, dist, device)
    ms_max = reduce_max(ms, dist, device)
    return total / (ms_max / 1000.0), ms_max


def gather_streams(q: float, scale: float, dist=None, device: str = "cpu") -> tuple[list, list]:
    """All ranks' (Q, scale), ordered by rank."""
    if dist is None or not dist.is_initialized():
        return [float(q)], [float(scale)]
    import torch
    t = torch.tensor([float(q), float(scale)], dtype=torch.float64, device=device)
    out = [torch.zeros_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(out, t)
    return [float(o[0]) for o in out], [float(o[1]) for o in out]
