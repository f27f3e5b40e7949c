"""The N > 1 path of bench.py: independent replicas whose step time is the
maximum over ranks.  Run with two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(10.0 + rank, dist, "cpu")
    finally:
        dist.destroy_process_group()


def test_step_time_is_max_over_two_gloo_ranks():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == 11.0 and out[1] == 11.0


def test_single_process_keeps_its_own_time():
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
