"""Replica plumbing for several GPUs: independent proofs shard across ranks
with no exchange on the data path; only the timing is reduced (the slowest
rank's time).  Works over NCCL (GPU ranks) and gloo (CPU ranks)."""
from __future__ import annotations


def rank_seed_base(rank: int) -> int:
    """First proof seed of a rank; ranks draw from disjoint ranges of 1000."""
    return 1000 * rank + 1


def shard(items, rank: int, world: int) -> list:
    """This rank's share of independent jobs (round robin)."""
    return list(items)[rank::world]


def _reduce(x: float, op: str) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(x: float) -> float:
    """The largest value over ranks (a job's time is the slowest replica's)."""
    return _reduce(x, "max")


def sum_over_ranks(x: float) -> float:
    return _reduce(x, "sum")


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
