"""Multi-rank host logic on CPU: world size 2 with the gloo backend.

Every rank computes the same problem assignment, the owned sets are disjoint
and cover all problems, and the timing / work reductions give the max and the
sum over ranks.  The GPU data path has no collective (problems are
independent), so nothing else crosses ranks.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

from femorph_b200 import shard


def test_assign_balances_and_is_deterministic():
    costs = [6 * n ** 3 * s for n, s in zip(range(8, 48, 3), range(100, 2000, 140))]
    a = shard.assign(costs, 4)
    assert a == shard.assign(costs, 4)
    loads = [sum(c for c, r in zip(costs, a) if r == k) for k in range(4)]
    assert max(loads) <= 1.35 * (sum(costs) / 4) or max(loads) == max(costs)
    assert sorted(i for k in range(4) for i in shard.mine(costs, 4, k)) == list(range(len(costs)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    owned = shard.mine(costs, world, rank)
    work = sum(costs[i] for i in owned)
    t = shard.reduce_max(1.0 + rank, dist)
    total = shard.reduce_sum(work, dist)
    import torch
    obj = [None] * world
    dist.all_gather_object(obj, owned)
    q.put((rank, owned, t, total, obj))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo():
    costs = [5, 9, 2, 7, 7, 3, 1, 8]
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    owned = [o[1] for o in out]
    assert not set(owned[0]) & set(owned[1])
    assert sorted(owned[0] + owned[1]) == list(range(len(costs)))
    for rank, _, t, total, gathered in out:
        assert t == 2.0  # max over ranks of (1 + rank)
        assert total == sum(costs)
        assert gathered == owned


def test_served_stream_draws_are_reproducible():
    from femorph_b200 import serve
    a = serve.request_params(16, seed=9)
    b = serve.request_params(16, seed=9)
    assert a == b
    ns = [x[0] for x in a]
    assert min(ns) >= 12 and max(ns) <= 64
