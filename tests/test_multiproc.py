"""Replica plumbing on two gloo ranks (CPU): max-over-ranks timing, request sharding, and
a rank that fails is reported to the others by a short process-group timeout rather than
a hang."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from jfli_b200 import replicas

    w, r, _ = replicas.init(backend="gloo", timeout_s=30)
    mine = replicas.shard(range(10), w, r)
    t = replicas.max_over_ranks(1.0 + r, device="cpu")
    n = replicas.sum_over_ranks(len(mine), device="cpu")
    replicas.barrier()
    q.put((r, mine, t, n))
    replicas.finalize()


def test_two_rank_replicas_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == [0, 2, 4, 6, 8] and out[1][1] == [1, 3, 5, 7, 9]
    assert all(o[2] == 2.0 for o in out)  # max over ranks
    assert all(o[3] == 10.0 for o in out)  # every request owned exactly once


def _failing_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from jfli_b200 import replicas

    replicas.init(backend="gloo", timeout_s=5)
    if rank == 1:
        os._exit(3)  # this rank leaves between steps without joining the collective
    try:
        replicas.max_over_ranks(1.0, device="cpu")
        q.put("no error")
    except Exception as e:  # the surviving rank must get an error, not hang
        q.put(type(e).__name__)


def test_lost_rank_surfaces_as_error_not_hang():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_failing_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert res != "no error"
