"""The N > 1 path of bench.py on CPU (gloo, world size 2).

The numeric phase does not shard: N GPUs run N independent replicas, and the job's time is the
slowest replica's. This is the one collective of that path, the max over ranks of the step time.
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank          # rank 1 is the slow replica
        out[rank] = bench.max_over_ranks(ms, dist, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2():
    world = 2
    out = mp.Manager().dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert dict(out) == {0: 15.0, 1: 15.0}
