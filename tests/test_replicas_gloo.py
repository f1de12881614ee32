"""The multi-GPU path of bench.py is independent replicas, one per rank,
timed as the slowest rank.  Its only cross-rank step, the max-over-ranks
reduction of the device timings, runs here on CPU with the gloo backend and
two ranks (no GPU), as the nccl process group does it on the box."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank            # rank 1 is the slowest
        ms_max = bench.max_over_ranks(ms, dist, "cpu")
        out[rank] = ms_max
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        assert out[0] == out[1] == 15.0


def test_max_over_ranks_single_process():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def _grad_rank(rank, world, port, out):
    import sys

    import numpy as np
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shots = bench.shots_of_rank(range(5), world, rank)
        # a stand-in gradient per shot: shot s contributes s + 1 everywhere
        g = np.zeros((3, 4, 5, 6), np.float32)
        for sh in shots:
            g += sh + 1
        total = bench.sum_over_ranks(g, dist, "cpu")
        out[rank] = (shots, float(total.min()), float(total.max()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_multi_shot_gradient_sum_gloo_two_ranks():
    """The multi-shot adjoint's host logic: shots split across two ranks,
    gradient volumes summed with one all-reduce."""
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_grad_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        assert out[0][0] == [0, 2, 4] and out[1][0] == [1, 3]
        assert out[0][1:] == out[1][1:] == (15.0, 15.0)
