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
