"""Independent replicas across ranks (the multi-GPU mode of this path).

The DG instances of the workloads are independent, so N GPUs run N replicas
with no data-path collective; the only cross-rank operations are the ones a
benchmark or a service needs for bookkeeping: a barrier, the maximum of the
per-rank times and the sum of the per-rank work.  Works with any
torch.distributed backend (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def rank_and_size():
    d = _dist()
    return (d.get_rank(), d.get_world_size()) if d else (0, 1)


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's replica (distinct per rank, reproducible)."""
    return int(base) * 1_000_003 + int(rank)


def _reduce(x: float, op_name: str, device=None) -> float:
    d = _dist()
    if d is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    d.all_reduce(t, op=getattr(d.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(x: float, device=None) -> float:
    return _reduce(x, "MAX", device)


def sum_over_ranks(x: float, device=None) -> float:
    return _reduce(x, "SUM", device)


def barrier() -> None:
    d = _dist()
    if d is not None:
        d.barrier()
