"""Multi-GPU runs are independent replicas (the single-rank drop-in has no
exchange step): bench.py's cross-rank reduction is checked here with two
gloo ranks on the CPU -- every rank gets the same whole-job number, bounded
by the slowest rank."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        seconds = [2.0, 3.0][rank]  # rank 1 is the slow one
        value, tmax = bench.replica_throughput(torch, dist, seconds, 1e6, 10, world, "cpu")
        out[rank] = (value, tmax)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_two_ranks():
    world = 2
    out = mp.get_context("spawn").Manager().dict()  # no fork of this process
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    for rank in range(world):
        value, tmax = out[rank]
        assert tmax == pytest.approx(3.0)
        assert value == pytest.approx(world * 1e6 * 10 / 3.0 / 1e9)


def test_replica_throughput_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    value, tmax = bench.replica_throughput(torch, None, 2.0, 1e6, 10, 1, "cpu")
    assert tmax == 2.0 and value == pytest.approx(1e6 * 10 / 2.0 / 1e9)
