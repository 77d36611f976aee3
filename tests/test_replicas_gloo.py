"""Multi-process (gloo, world_size 2, CPU) checks of the replica plumbing used
by bench.py under torchrun: timing reduction, aggregate throughput, sharding
of independent units and per-rank seeds."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from pde_solver_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    dist = replicas.init("gloo", timeout_s=60)
    try:
        w, r, l = replicas.rank_env()
        ms = 100.0 + 50.0 * r  # rank 1 is the slow one
        dist.barrier()
        m = replicas.max_over_ranks(ms, dist)
        rate = replicas.aggregate_rate(w, 10, m)
        mine = list(replicas.shard(2304, w, r))
        q.put((r, w, m, rate, mine[0], mine[-1], len(mine), replicas.replica_seed(1234, r)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_plumbing_world2():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r, w, m, rate, first, last, count, seed in out:
        assert w == 2 and m == 150.0
        assert rate == pytest.approx(2 * 10 / 0.150)
        assert seed == 1234 + r
    assert out[0][4] == 0 and out[0][5] + 1 == out[1][4] and out[1][5] == 2303
    assert out[0][6] + out[1][6] == 2304



def test_shard_covers_every_unit_once():
    for count in (0, 1, 7, 2304):
        for world in (1, 2, 3, 8):
            seen = [u for r in range(world) for u in replicas.shard(count, world, r)]
            assert seen == list(range(count))


def test_single_process_is_identity():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.aggregate_rate(1, 10, 1000.0) == pytest.approx(10.0)
