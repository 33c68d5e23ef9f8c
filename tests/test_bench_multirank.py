"""bench.py's multi-rank path on the CPU: two gloo ranks, each with its own
measured time; the reported time is the slowest rank's and the whole-job
throughput counts both replicas (replicas only: no data-path collective)."""
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


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    my_ms = [120.0, 80.0][rank]
    ms_max = bench.max_over_ranks(torch, my_ms, "cpu", world)
    value = bench.whole_job_gops(world, 2.0 * 8192 ** 3, 10, ms_max)
    out[rank] = (ms_max, value)
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
    assert out[0][0] == out[1][0] == 120.0
    want = 2 * 2.0 * 8192 ** 3 * 10 / 0.120 / 1e9
    assert abs(out[0][1] - want) < 1e-6 * want
    assert out[0][1] == out[1][1]


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(torch, 3.5, "cpu", 1) == 3.5
