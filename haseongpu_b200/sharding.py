"""Sample-range sharding over ranks (one process per GPU).

The backward method treats every sample point independently, so N GPUs split
the sample range into contiguous shards and need no collective on the data
path; only the per-sample results are gathered once at the end.  This
replaces the reference's MPI sample distribution (the legacy ``mapIdx`` of
include/core/haseWorker.hpp:27-37 strides work over workers the same way).
"""

from __future__ import annotations

import numpy as np

RESULT_FIELDS = ("phiAse", "standardError", "relativeStandardError", "totalRays", "dndtAse", "droppedRays")


def shard_range(first: int, last: int, world: int, rank: int) -> tuple[int, int]:
    """Inclusive [first, last] split into `world` contiguous shards; empty shards are (x, x-1)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    n = last - first + 1
    if n < 0:
        raise ValueError("empty range")
    base, extra = divmod(n, world)
    lo = first + rank * base + min(rank, extra)
    size = base + (1 if rank < extra else 0)
    return lo, lo + size - 1


def gather_results(local: dict, first: int, last: int, group=None, device=None) -> dict:
    """All-gather per-rank result arrays (torch.distributed; gloo on CPU tensors,
    NCCL on ``device`` tensors) into full [first, last] arrays on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    n = last - first + 1
    out = {}
    for name in RESULT_FIELDS:
        a = np.asarray(local[name])
        t = torch.from_numpy(a.astype(np.float64))
        sizes = [shard_range(first, last, world, r) for r in range(world)]
        width = max(hi - lo + 1 for lo, hi in sizes)
        buf = torch.zeros(width, dtype=torch.float64, device=device)
        buf[: t.numel()] = t.to(buf.device)
        parts = [torch.zeros(width, dtype=torch.float64, device=device) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
        full = np.concatenate([p[: hi - lo + 1].cpu().numpy() for p, (lo, hi) in zip(parts, sizes)])
        assert full.size == n
        out[name] = full.astype(a.dtype)
    return out


def shard_media(costs, world: int, rank: int | None = None):
    """Media of a batched solve spread over `world` ranks: longest-first greedy
    assignment by cost (e.g. sample points x prisms x expected rays), ties to
    the lowest rank, deterministic on every rank.  Returns the owner rank of
    every medium, or the indices of `rank`'s media (in increasing order)."""
    if world <= 0 or (rank is not None and not 0 <= rank < world):
        raise ValueError("need world > 0 and 0 <= rank < world")
    costs = np.asarray(costs, np.float64)
    if np.any(costs < 0) or not np.all(np.isfinite(costs)):
        raise ValueError("costs must be finite and non-negative")
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world)
    owner = np.empty(costs.size, np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    return owner if rank is None else np.nonzero(owner == rank)[0]


def gather_media_results(local: dict, count: int, group=None) -> list:
    """All-gather per-medium results ({medium index: result dict of arrays})
    from every rank into one list of `count` entries on every rank."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, {int(k): {f: np.asarray(v) for f, v in r.items()} for k, r in local.items()},
                           group=group)
    out = [None] * count
    for p in parts:
        for k, r in p.items():
            if out[k] is not None:
                raise ValueError(f"medium {k} was solved on two ranks")
            out[k] = r
    missing = [k for k, r in enumerate(out) if r is None]
    if missing:
        raise ValueError(f"media {missing} were solved on no rank")
    return out
