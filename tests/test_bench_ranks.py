"""bench.py's multi-GPU arithmetic (replicas, one process per GPU) on two gloo ranks on the CPU:
the job time is the slowest rank's, the event count the sum over ranks."""
import os
import socket
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, ev = bench.combine_over_ranks(1.5 + rank, 1000.0 * (rank + 1), world, "cpu")
        out[rank] = (ms, ev)
    finally:
        dist.destroy_process_group()


def test_combine_over_ranks_two_gloo_ranks():
    world = 2
    out = mp.Manager().dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert out[0] == out[1] == (2.5, 3000.0)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.combine_over_ranks(3.0, 7.0, 1, "cpu") == (3.0, 7.0)
