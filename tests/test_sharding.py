"""Multi-process (world size 2, gloo, CPU) tests of the instance-sharding host logic that
``bench.py --gpus N`` and multi-GPU users rely on: every instance is owned by exactly one
rank, timings reduce to the maximum over ranks, and results gather back in order."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dynamiqs_b200.sharding import gather_to, max_over_ranks, shard_range, sharded_solve


@pytest.mark.parametrize('batch', [0, 1, 7, 4096])
@pytest.mark.parametrize('world', [1, 2, 3, 8])
def test_shard_range_partitions(batch, world):
    owned = np.zeros(batch, int)
    sizes = []
    for r in range(world):
        a, b = shard_range(batch, r, world)
        owned[a:b] += 1
        sizes.append(b - a)
    assert np.all(owned == 1)
    assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        # a fake solver: per-instance "result" = 10 * index, time = rank-dependent
        items = np.arange(11)
        start, stop, res = sharded_solve(lambda blk: torch.tensor(blk * 10.0), items, rank, world)
        t = max_over_ranks(1.0 + rank)
        full = gather_to(res, dst=0)
        if rank == 0:
            q.put((t, full.tolist()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    t, full = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert t == 2.0
    assert full == [10.0 * i for i in range(11)]
