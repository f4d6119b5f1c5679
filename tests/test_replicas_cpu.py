"""The multi-GPU path of bench.py is N independent replicas (no collective on
the data path); its host logic -- rank discovery, barrier, max-over-ranks
timing -- runs here as two gloo processes on the CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w, r, loc = bench.dist_setup(None)
        assert (w, r, loc) == (world, rank, rank)
        bench.barrier(world)
        # each rank reports its own step time; every rank must see the maximum
        t = bench.max_over_ranks(10.0 + rank, world, torch.device("cpu"))
        out[rank] = t
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_replicas_agree_on_the_max_time():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        assert dict(out) == {0: 11.0, 1: 11.0}


def test_single_process_needs_no_process_group():
    assert bench.max_over_ranks(3.5, 1, torch.device("cpu")) == 3.5
    bench.barrier(1)
