"""Multi-GPU form: replicas only.

Stars are independent, so N GPUs run N independent replicas of the batched
engine on disjoint star shards (one process per GPU, launched by
torch.distributed.run).  The only collectives are host-side: a barrier
around the timed region, the max over ranks of the device time, and a
gather of results.  Nothing on the data path is exchanged between GPUs.
"""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous, balanced share of n_items for this rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank/world")
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return range(lo, lo + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, device=None) -> float:
    """Max of a float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_to_rank0(obj):
    """Gather a picklable object from every rank on rank 0 (list by rank), None elsewhere."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
