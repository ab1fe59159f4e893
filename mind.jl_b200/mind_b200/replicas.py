"""Multi-GPU runs: one process per GPU, each advancing its own network replica.

The per-step loop has no exchange between GPUs when every rank simulates an
independent network, so ranks only meet to time the run: the whole-job figure
is the units all ranks processed divided by the slowest rank's device time
(max over ranks).  Replicas differ only in the build! seed (NetStim streams).
"""
from __future__ import annotations


def replica_seed(base_seed: int, rank: int) -> int:
    return int(base_seed) + int(rank)


def reduce_timing(run_ms: float, units: float, device=None):
    """(max run_ms over ranks, sum of units over ranks); identity without a process group."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(run_ms), float(units)
    t = torch.tensor([run_ms], dtype=torch.float64, device=device)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())
