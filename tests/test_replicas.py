"""Replica plumbing on CPU (gloo, two ranks): disjoint stream shards, the
aggregate of pixels and the max of device times, and a failing rank turning
into an error on the survivor's collective instead of a hang."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from wema_b200 import replicas


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shards_are_disjoint_and_complete():
    items = list(range(48))
    parts = [replicas.shard(items, r, 4) for r in range(4)]
    assert sorted(x for p in parts for x in p) == items
    assert all(len(p) == 12 for p in parts)
    with pytest.raises(ValueError):
        replicas.shard(items, 4, 4)


def _rank_ok(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist = replicas.init("gloo", timeout_s=30)
    mine = replicas.shard(range(10), rank, world)
    pix, ms, rate = replicas.aggregate(100.0 * len(mine), 2.0 + rank, dist)
    q.put((rank, mine, pix, ms, rate))
    dist.destroy_process_group()


def test_aggregate_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank_ok, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0][1] == [0, 2, 4, 6, 8] and got[1][1] == [1, 3, 5, 7, 9]
    for _, _, pix, ms, rate in got:
        assert pix == 1000.0 and ms == 3.0                   # sum of pixels, max of times
        assert abs(rate - 1000.0 / 3e-3 / 1e6) < 1e-12


def _rank_fail(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist = replicas.init("gloo", timeout_s=5)
    if rank == 1:
        q.put((rank, "left"))
        q.close()
        q.join_thread()                                     # the message is out before the exit
        os._exit(0)                                         # leaves between steps, no collective
    try:
        replicas.aggregate(1.0, 1.0, dist)
        q.put((rank, "no error"))
    except Exception as ex:                                 # the collective times out / breaks
        q.put((rank, "error:" + type(ex).__name__))


def test_dead_rank_is_an_error_not_a_hang():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank_fail, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert got[1] == "left"
    assert got[0].startswith("error:")
