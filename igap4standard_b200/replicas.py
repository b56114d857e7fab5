"""Multi-GPU use of the assembly: replicas and instance sharding.

One mesh never spans GPUs here (its 64^3 working set is ~4 GB of a B200's
180 GB), so the path does not shard: N processes run N independent meshes,
and a batch of independent instances is split across ranks without any
data-path collective.  The only collective is the max-over-ranks of a timing.
"""
import os


def rank_world():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def shard(n_items, rank, world):
    """Contiguous, balanced slice [lo, hi) of n_items for this rank."""
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def max_over_ranks(value, device=None):
    """Max of a float over the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
