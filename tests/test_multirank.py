"""Multi-process host logic on CPU (gloo, world size 2): the bench's
max-over-ranks timing, and the replica rule that each rank runs its own
library context and only rank 0 reports."""

import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms = bench.max_over_ranks(1.0 + rank * 2.5, world, torch.device("cpu"))
        single = bench.max_over_ranks(7.0, 1, torch.device("cpu"))
        results[rank] = (ms, single)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as manager:
        results = manager.dict()
        mp.start_processes(_worker, args=(world, port, results), nprocs=world,
                           start_method="spawn", join=True)
        got = dict(results)
    assert got == {0: (3.5, 7.0), 1: (3.5, 7.0)}
