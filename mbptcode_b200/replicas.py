"""Independent replicas over ranks (one process per GPU).

The route does not shard in this build: a system's chi0 -> W -> Sigma sweep
runs on one GPU. What spreads over GPUs is independent work -- separate
systems (the learned warm start's training set) or repeated sweeps -- with
no collective on the data path. This module holds the host logic of that:
which rank takes which systems, the job time as the maximum over ranks, and
the gathering of per-rank results (small host objects) at the end.
"""
from __future__ import annotations


def shard(n_items, rank, world):
    """Items of this rank: rank, rank + world, ... (round robin)."""
    if not 0 <= rank < world:
        raise ValueError(f'rank {rank} outside a world of {world}')
    return list(range(rank, n_items, world))


def max_over_ranks(value, group=None, device=None):
    """The largest `value` over the ranks of `group` (the value itself
    without torch.distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather(obj, group=None):
    """Every rank's `obj`, in rank order, on every rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, obj, group=group)
    return out
