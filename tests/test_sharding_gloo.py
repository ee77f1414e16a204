"""Multi-rank host logic on CPU: sample-range shards cover the range exactly
once and the result all-gather (gloo, world size 2 and 3) reassembles them."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest


def test_shard_range_partitions():
    from haseongpu_b200.sharding import shard_range

    for first, last in [(0, 0), (0, 9), (5, 4213), (3, 4)]:
        for world in (1, 2, 3, 8):
            covered = []
            for r in range(world):
                lo, hi = shard_range(first, last, world, r)
                covered.extend(range(lo, hi + 1))
            assert covered == list(range(first, last + 1))
    with pytest.raises(ValueError):
        shard_range(0, 9, 2, 2)


def _fake_solve(lo, hi):
    s = np.arange(lo, hi + 1)
    return {"phiAse": (1.5 * s).astype(np.float32), "standardError": 0.1 * s, "relativeStandardError": 1.0 / (s + 1),
            "totalRays": (1000 + s).astype(np.uint32), "dndtAse": -2.0 * s, "droppedRays": (s % 3).astype(np.uint32)}


def _worker(rank, world, port, first, last, q):
    import torch.distributed as dist

    from haseongpu_b200.sharding import gather_results, shard_range

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lo, hi = shard_range(first, last, world, rank)
        full = gather_results(_fake_solve(lo, hi), first, last)
        expect = _fake_solve(first, last)
        ok = all(np.array_equal(full[k], expect[k]) for k in expect)
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gather_results_gloo(world):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, 7, 1030, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    results = dict(q.get(timeout=10) for _ in range(world))
    assert all(results.values()) and len(results) == world


def test_shard_media_covers_every_medium_once_and_balances():
    from haseongpu_b200.sharding import shard_media

    rng = np.random.default_rng(3)
    costs = np.exp(rng.uniform(np.log(200), np.log(20000), 64)) * rng.integers(5, 41, 64)
    for world in (1, 2, 3, 8):
        owner = shard_media(costs, world)
        assert owner.shape == (64,) and set(owner) <= set(range(world))
        parts = [shard_media(costs, world, r) for r in range(world)]
        assert sorted(np.concatenate(parts).tolist()) == list(range(64))
        loads = np.array([costs[p].sum() for p in parts])
        # longest-first greedy: no rank exceeds the mean by more than the largest medium
        assert loads.max() <= costs.sum() / world + costs.max()
    with pytest.raises(ValueError):
        shard_media(costs, 2, 2)
    with pytest.raises(ValueError):
        shard_media([-1.0], 1)


def _fake_medium(k):
    return {"phiAse": np.full(3 + k % 4, k, np.float32), "totalRays": np.arange(3 + k % 4, dtype=np.uint32) + k}


def _media_worker(rank, world, port, q):
    import torch.distributed as dist

    from haseongpu_b200.sharding import gather_media_results, shard_media

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = np.arange(1, 17, dtype=np.float64) ** 2
        mine = shard_media(costs, world, rank)
        full = gather_media_results({int(k): _fake_medium(int(k)) for k in mine}, 16)
        ok = all(np.array_equal(full[k][f], _fake_medium(k)[f]) for k in range(16) for f in ("phiAse", "totalRays"))
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


def test_gather_media_results_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_media_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    results = dict(q.get(timeout=10) for _ in range(2))
    assert all(results.values()) and len(results) == 2
