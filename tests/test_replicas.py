"""Replica path on two gloo ranks (CPU): disjoint job shards and seed ranges,
and the timing reduction the bench uses (the slowest rank's time)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from virgo_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = replicas.shard(range(10), rank, world)
        t = replicas.max_over_ranks(1.0 + rank)
        n = replicas.sum_over_ranks(len(jobs))
        replicas.barrier()
        q.put((rank, jobs, replicas.rank_seed_base(rank), t, n))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, j0, s0, t0, n0), (r1, j1, s1, t1, n1) = out
    assert sorted(j0 + j1) == list(range(10)) and not set(j0) & set(j1)
    assert abs(s0 - s1) >= 1000                     # disjoint seed ranges
    assert t0 == t1 == 2.0 and n0 == n1 == 10.0     # max of times, total of jobs


def test_single_process_needs_no_group():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.shard([1, 2, 3], 0, 1) == [1, 2, 3]
