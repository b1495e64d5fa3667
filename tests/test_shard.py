"""CPU, world size 2 over gloo: limb sharding, the max-over-ranks timing and
the union of per-rank results (computed with the oracle round trip) equal
to the single-process result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from axhel_b200.shard import max_over_ranks, shard_range


def test_shard_ranges_cover_and_align():
    for count, L in ((768, 24), (48, 24), (24, 24), (96, 3)):
        for world in (1, 2, 3, 4, 8):
            ranges = [shard_range(count, L, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == count
            for (a, b), (c, d) in zip(ranges, ranges[1:]):
                assert b == c
            assert all(a % L == 0 and b % L == 0 and b >= a for a, b in ranges)
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= L
    with pytest.raises(ValueError):
        shard_range(100, 24, 0, 2)
    with pytest.raises(ValueError):
        shard_range(48, 24, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, L, count, out):
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    from pyoracle import Oracle

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    o = Oracle()
    qs = [o.find_ntt_prime_near(n, 40 + i, 1, 2) for i in range(L)]
    tabs = [o.tables(n, q, o.find_primitive_root(n, q)) for q in qs]
    st = o.rng(77)
    data = np.concatenate([o.random_vector(st, n, qs[i % L]) for i in range(count)])
    b, e = shard_range(count, L, rank, world)
    res = []
    for i in range(b, e):
        k = i % L
        x = data[i * n:(i + 1) * n]
        lazy = o.forward(x, qs[k], tabs[k][0], 1, 4)
        res.append(lazy)
        assert np.array_equal(o.inverse(o.reduce(lazy, qs[k], 4, 2), qs[k], tabs[k][1], tabs[k][2], 2, 1), x)
    mine = np.concatenate(res) if res else np.zeros(0, np.uint64)
    gathered = [None] * world
    dist.all_gather_object(gathered, (b, e, mine))
    t = max_over_ranks(float(rank + 1), dist)
    if rank == 0:
        full = np.concatenate([g[2] for g in sorted(gathered, key=lambda g: g[0])])
        ref = np.concatenate([o.forward(data[i * n:(i + 1) * n], qs[i % L], tabs[i % L][0], 1, 4)
                              for i in range(count)])
        out.put((bool(np.array_equal(full, ref)), t))
    dist.destroy_process_group()


def test_two_rank_gloo_shards_match_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, 256, 3, 9, q)) for r in range(2)]
    for p in procs:
        p.start()
    ok, t = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert ok
    assert t == 2.0
