"""The multi-GPU path of bench.py is N independent replicas whose only exchange is the
job time (the max over ranks) and barriers; this runs that exchange on CPU with gloo,
two ranks, the way torchrun launches bench.py (127.0.0.1 rendezvous)."""
import os
import socket
import sys

import pytest
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
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    assert bench.dist_info() == (rank, rank, world)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        # rank r reports 10 + r ms: every rank must see the slowest rank's time
        out[rank] = bench.max_over_ranks(dist, 10.0 + rank, device="cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    assert dict(out) == {0: 11.0, 1: 11.0}


def test_single_process_needs_no_exchange():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.5) == 3.5


def _shard_rank(rank, world, port, sizes, out):
    sys.path.insert(0, ROOT)
    import within_b200 as wb
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = wb.shard_problems(sizes, world)[rank]
        got = [None] * world
        dist.all_gather_object(got, (mine, sum(sizes[i] for i in mine)))
        out[rank] = got
    finally:
        dist.destroy_process_group()


def _sizes(n=256, seed=0):
    import numpy as np
    # the uneven batch's observation counts: log-uniform on [1e3, 1e6]
    return [int(v) for v in np.exp(np.random.default_rng(seed).uniform(np.log(1e3), np.log(1e6), n))]


def test_shard_problems_covers_every_problem_once_and_balances():
    sys.path.insert(0, ROOT)
    import within_b200 as wb
    sizes = _sizes()
    for world in (1, 2, 3, 4, 8):
        shards = wb.shard_problems(sizes, world)
        assert len(shards) == world
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in s) for s in shards]
        # greedy largest-first: no rank exceeds the mean by more than one problem
        assert max(loads) <= sum(sizes) / world + max(sizes)
    with pytest.raises(ValueError):
        wb.shard_problems(sizes, 0)


def test_independent_problems_shard_over_two_gloo_ranks():
    """Each rank of `bench.py --workload uneven` under torchrun takes its shard with no
    exchange: the two ranks' shards are disjoint, cover the batch, and agree with the
    single-process assignment."""
    sys.path.insert(0, ROOT)
    import within_b200 as wb
    world, port, sizes = 2, _free_port(), _sizes(seed=3)
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_shard_rank, args=(world, port, sizes, out), nprocs=world, join=True, start_method="spawn")
    assert out[0] == out[1]
    shards = [s for s, _ in out[0]]
    assert sorted(i for s in shards for i in s) == list(range(len(sizes)))
    assert shards == wb.shard_problems(sizes, world)
    loads = [l for _, l in out[0]]
    assert max(loads) - min(loads) <= max(sizes)
