"""Multi-GPU plumbing of the path: replicas, no data-path collective.

Every sample is a pure function of (request seed, pixel, sample index)
(src/pathtrace.rs:45-86), so work shards across GPUs with no exchange:
frames, requests, or row bands of one frame go to ranks independently, and
the only collectives are host-side bookkeeping (a barrier around timed
regions and the max of the ranks' device times). torch.distributed carries
them (NCCL between GPUs, gloo on CPU hosts).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple, TypeVar

T = TypeVar("T")


def shard(items: Sequence[T], rank: int, world: int) -> List[T]:
    """Round-robin share of `items` for `rank` of `world`: disjoint across
    ranks, together exactly `items`, stable in order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    return list(items[rank::world])


def row_bands(height: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous rows [first, end) of a frame for `rank`: balanced to one
    row, covering the frame once across ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    base, extra = divmod(height, world)
    first = rank * base + min(rank, extra)
    return first, first + base + (1 if rank < extra else 0)


def max_over_ranks(x: float, device=None) -> float:
    """Max of `x` over the default process group (the job's time is its
    slowest rank's); `x` itself when no group is initialised."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device=None) -> float:
    """Sum of `x` over the default process group (units all ranks processed)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
