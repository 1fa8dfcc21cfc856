"""Multi-process host logic on the CPU: two gloo ranks on 127.0.0.1 shard a
batch of instances, time with the max over ranks and gather per-instance
results in rank order (the N>1 path of bench.py and of sharded batches)."""
import os
import socket

import numpy as np
import pytest

from airtoolsii_b200 import dist as D


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        cost = np.arange(1, 12, dtype=float) ** 2
        own = D.shard(11, rank, world, cost)
        t = D.max_over_ranks(1.5 + rank)
        tot = D.sum_over_ranks(float(len(own)))
        # per-instance results: (instance index, rank, 2*index)
        local = np.stack([own, np.full(own.size, rank), 2.0 * own], axis=1) if own.size else np.zeros((0, 3))
        allr = D.gather_units(local)
        q.put((rank, own.tolist(), t, tot, allr.tolist()))
    finally:
        dist.destroy_process_group()


def test_shard_covers_every_unit_once():
    for n in (0, 1, 7, 512):
        for world in (1, 2, 3, 8):
            parts = [D.shard(n, r, world) for r in range(world)]
            assert np.array_equal(np.concatenate(parts), np.arange(n))
            sizes = [p.size for p in parts]
            assert max(sizes) - min(sizes) <= 1
            cost = np.random.default_rng(n).random(n) * 10
            parts = [D.shard(n, r, world, cost) for r in range(world)]
            assert np.array_equal(np.concatenate(parts), np.arange(n))


def test_shard_balances_cost():
    cost = np.r_[np.full(100, 1.0), np.full(10, 100.0)]
    a, b = (D.shard(110, r, 2, cost) for r in range(2))
    ca, cb = cost[a].sum(), cost[b].sum()
    assert abs(ca - cb) <= cost.max()
    with pytest.raises(ValueError):
        D.shard(5, 2, 2)


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    owns = [o[1] for o in out]
    assert sorted(owns[0] + owns[1]) == list(range(11))
    assert all(o[2] == 2.5 for o in out)             # max over ranks of 1.5 + rank
    assert all(o[3] == 11.0 for o in out)            # every instance counted once
    for o in out:                                    # rank-ordered gather, same on both ranks
        rows = np.array(o[4])
        assert np.array_equal(rows[:, 0], np.arange(11))
        assert np.array_equal(rows[:, 2], 2 * np.arange(11))
        assert np.array_equal(rows[:, 1], [0] * len(owns[0]) + [1] * len(owns[1]))
