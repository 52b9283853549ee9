"""Multi-GPU plumbing of the path: replicas, no data-path collective.

Every sample is a pure function of (request seed, pixel, sample index)
(src/pathtrace.rs:45-86), so work shards across GPUs with no exchange:
frames, requests, or row bands of one frame go to ranks independently.
Serving shards whole requests with scene affinity (plan_requests: each
GPU keeps its own scene cache) and collects the images in request order
on one rank (gather_ordered). The only collectives are host-side
bookkeeping: that gather, a barrier around timed regions and the max of the
ranks' device times. torch.distributed carries them (NCCL between GPUs,
gloo on CPU hosts).
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple, TypeVar

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


def plan_requests(scene_keys: Sequence[int], work: Sequence[float], world: int) -> List[int]:
    """Owner rank of each request for serving on `world` GPUs, each with its
    own resident scene cache: all requests of one scene go to one rank (a
    scene is uploaded to one GPU only), and scenes are dealt largest total
    work first to the least-loaded rank (greedy longest-processing-time
    balancing). Deterministic: ties go to the lower scene key / rank."""
    if world < 1:
        raise ValueError(f"world {world}")
    if len(scene_keys) != len(work):
        raise ValueError("one work estimate per request")
    per_scene: Dict[int, float] = {}
    for k, w in zip(scene_keys, work):
        per_scene[k] = per_scene.get(k, 0.0) + float(w)
    load = [0.0] * world
    owner_of: Dict[int, int] = {}
    for k in sorted(per_scene, key=lambda k: (-per_scene[k], k)):
        r = min(range(world), key=lambda i: (load[i], i))
        owner_of[k] = r
        load[r] += per_scene[k]
    return [owner_of[k] for k in scene_keys]


def gather_ordered(results: Dict[int, T], n: int, dst: int = 0) -> Optional[List[T]]:
    """The results of every rank's share of `n` requests (request index ->
    result), in request order, on rank `dst` (None on the others). Every
    index must be produced by exactly one rank. Without a process group the
    local results are the whole set."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        parts = [results]
        rank = dst
    else:
        rank = dist.get_rank()
        parts = [None] * dist.get_world_size() if rank == dst else None
        dist.gather_object(results, parts, dst=dst)
    if rank != dst:
        return None
    merged: Dict[int, T] = {}
    for part in parts:
        for i, v in part.items():
            if i in merged:
                raise ValueError(f"request {i} was produced twice")
            merged[i] = v
    missing = [i for i in range(n) if i not in merged]
    if missing:
        raise ValueError(f"requests {missing[:5]} were produced by no rank")
    return [merged[i] for i in range(n)]


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
