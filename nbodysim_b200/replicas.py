"""Replica timing across ranks (one process per GPU, independent replicas).

The Barnes-Hut path of this engine runs one system per GPU; several GPUs run
independent replicas with no collective on the data path. Only the timing
needs ranks to agree: every rank times its own steps on the device, the job's
time is the slowest rank's, and the work is the sum over ranks.
"""
from __future__ import annotations


def job_totals(dist, device, ms: float, units: float) -> tuple[float, float]:
    """(max over ranks of `ms`, sum over ranks of `units`); identity without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms), float(units)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())
