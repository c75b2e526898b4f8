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
