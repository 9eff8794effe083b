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


def _shard_rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    import importlib
    pkg = ge.load_package()
    cfgs = importlib.import_module(pkg.__name__ + ".configs")
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = __import__("numpy").random.default_rng(3)
        grids = cfgs.ENSEMBLE_GRIDS
        sims = [dict(dims=grids[int(k)][0], nslots=65536) for k in rng.integers(0, len(grids), 64)]
        mine = cfgs.shard([cfgs.sim_cost(s) for s in sims], world)[rank]
        # every rank's view of the whole split, gathered from the ranks
        mask = torch.zeros(64, dtype=torch.int64)
        mask[mine] = rank + 1
        views = [torch.zeros(64, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(views, mask)
        total = sum(views)
        out[rank, :64] = total
        out[rank, 64] = sum(cfgs.sim_cost(sims[i]) for i in mine)
        out[rank, 65] = max(cfgs.sim_cost(s) for s in sims)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_the_ensemble():
    """configs.shard gives the two ranks disjoint simulation sets that cover
    the ensemble, with loads within one simulation's cost of each other."""
    world = 2
    out = torch.zeros((world, 66), dtype=torch.int64).share_memory_()
    mp.spawn(_shard_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        # each simulation is owned by exactly one rank (values 1 or 2, never 0 or 3)
        assert set(out[r, :64].tolist()) <= {1, 2}
        assert torch.equal(out[r, :64], out[0, :64])
    assert abs(int(out[0, 64]) - int(out[1, 64])) <= int(out[0, 65])


def test_shard_is_balanced_and_deterministic():
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    import importlib
    pkg = ge.load_package()
    cfgs = importlib.import_module(pkg.__name__ + ".configs")
    costs = [7, 3, 3, 9, 1, 5, 5, 2]
    for world in (1, 2, 3, 8, 10):
        parts = cfgs.shard(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
        assert parts == cfgs.shard(costs, world)
    with pytest.raises(ValueError):
        cfgs.shard(costs, 0)
