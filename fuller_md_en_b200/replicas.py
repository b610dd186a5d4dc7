"""Independent replicas across ranks (one process per GPU): the path has no
exchange step, so ranks share nothing but the timing reduction.  Works with
the NCCL backend on GPUs and with gloo on CPU (tests)."""
from __future__ import annotations


def replica_seed(base: int, rank: int) -> int:
    """Each rank advances its own system, seeded from the base seed."""
    return base + rank


def max_over_ranks(ms: float, device=None) -> float:
    """Largest per-rank duration (ms): the job finishes when its slowest
    replica does.  Single process: returns ms unchanged."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(ms)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: int, steps: int, ms_max: float, world_size: int) -> float:
    """Whole-job units x steps per second over all ranks (weak scaling: every
    rank has the same work)."""
    return world_size * units_per_rank * steps / (ms_max / 1e3)
