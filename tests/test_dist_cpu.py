"""The bench's multi-rank path on CPU: gloo, world size 2.  Replicas run independent work; the
only collectives are the max-over-ranks time and the sum of work units."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        # rank r "processes" 100 units per step for 4 steps in (r + 1) seconds
        value, t_max = bench.replica_throughput(100, 4, float(rank + 1), dist, 'cpu')
        q.put((rank, value, t_max))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_is_total_work_over_slowest_rank():
    world = 2
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, t_max in res:
        assert t_max == 2.0
        assert value == pytest.approx(100 * 4 * world / 2.0)


def test_single_process_needs_no_collective():
    value, t = bench.replica_throughput(10, 3, 1.5, None)
    assert t == 1.5 and value == pytest.approx(20.0)
