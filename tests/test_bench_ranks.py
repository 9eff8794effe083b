"""The multi-rank path of bench.py on CPU: two gloo ranks (one process per
GPU on a box) agree on the max-over-ranks timing and on the whole-job rate
of N independent replicas."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 3.0 * rank          # rank 1 is the slow one
        m = bench.rank_max(ms, world, "cpu")
        dist.barrier()
        out[rank] = m
        out[world + rank] = bench.whole_job_rate(100, m, world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    world = 2
    out = torch.zeros(2 * world, dtype=torch.float64).share_memory_()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1] == 13.0
    assert out[2] == out[3] == pytest.approx(2 * 100 / 0.013)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.rank_max(7.5, 1, "cpu") == 7.5
    assert bench.whole_job_rate(50, 25.0, 1) == pytest.approx(2000.0)
