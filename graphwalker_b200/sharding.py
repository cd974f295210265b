"""Multi-GPU plumbing of the walk workload (one process per GPU).

With counter-based draws every walk is independent, so the path shards by
walk: the graph is replicated on each GPU and each rank runs its own walks.
Weak scaling gives rank r the walk ids [r * n, (r + 1) * n) of an n-walk set
per rank; strong scaling splits one walk set into contiguous ranges.  The one
exchange of the path is the sum of the per-vertex visit counters (u32,
wrapping like the device counters), done with a single all-reduce.
"""
from __future__ import annotations


def walk_id_offset(rank: int, walks_per_rank: int) -> int:
    """First walk id of `rank` under weak scaling."""
    return rank * walks_per_rank


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Walks [lo, hi) of `rank` when `total` walks are split over `world` ranks."""
    base, extra = divmod(total, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def reduce_counts(counts, group=None):
    """Sums int32 visit counters over all ranks in place (one all-reduce)."""
    import torch.distributed as dist
    dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
    return counts


def max_over_ranks(value: float, device=None, group=None) -> float:
    """The slowest rank's time: every multi-GPU number is reported this way."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
