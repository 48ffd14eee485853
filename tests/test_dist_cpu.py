"""The multi-GPU timing logic of bench.py on two CPU processes (gloo): every rank waits at the barriers and
reports the slowest rank's time, and the replica throughput counts the units of every rank.  (On GPUs the
same functions run over NCCL, one process per GPU, with no collective on the data path.)"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        ms = 10.0 * (rank + 1)               # rank 1 is the slow one
        out[rank] = bench.max_over_ranks(ms, world)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_on_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        assert dict(out) == {0: 20.0, 1: 20.0}


def test_single_rank_needs_no_process_group():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    bench.barrier(1)
    assert bench.max_over_ranks(3.5, 1) == 3.5
