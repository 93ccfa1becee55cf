"""The N>1 plumbing of bench.py on the CPU: with --gpus N the bench runs N independent replicas of the
single-GPU workload (the solve does not shard across GPUs), so the only cross-rank steps are the barrier
and the max-over-ranks timing.  Two gloo ranks check that reduction, and that the reference arm does no
work on ranks other than 0."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        # rank r reports (r + 1) * 10 ms: every rank must see the slowest, 20 ms
        out[rank] = bench.max_over_ranks((rank + 1) * 10.0, dist, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    assert dict(out) == {0: 20.0, 1: 20.0}


def test_reference_arm_other_ranks_do_nothing():
    import argparse

    import bench

    args = argparse.Namespace(steps=1, warmup=1, gpus=2)
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.run_reference_arm(args, rank=1, world=2) == 0
    assert buf.getvalue() == ""
