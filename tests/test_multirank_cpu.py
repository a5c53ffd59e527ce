"""The bench's multi-GPU path on CPU: two ranks over the gloo backend.

With N GPUs the bench runs N independent replicas of the workload (the grid
is not decomposed, there is no data-path collective); each rank times its own
replica and the job is timed by the slowest rank.  These tests run that
reduction and the reference arm's rank rule with world_size 2 on CPU."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        own = [3.0, 5.0][rank]                      # this rank's replica time, s
        worst = bench.max_over_ranks(own, dist, torch, "cpu")
        rate = bench.aggregate_rate(world, 1000, 10, worst)
        # the reference arm prints on rank 0 only; other ranks return silently
        class A:
            steps, warmup, ref_steps, workload = 1, 0, 1, "fm_demag"
        buf = io.StringIO()
        if rank != 0:
            with redirect_stdout(buf):
                bench.run_reference_arm(A, rank, world)
        dist.barrier()
        out[rank] = (worst, rate, buf.getvalue())
    finally:
        dist.destroy_process_group()


def test_replicas_are_timed_by_the_slowest_rank():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert sorted(out.keys()) == [0, 1]
    for r in range(world):
        worst, rate, printed = out[r]
        assert worst == 5.0
        assert rate == pytest.approx(2 * 1000 * 10 / 5.0)
    assert out[1][2] == ""


def test_aggregate_rate_without_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(2.5, None, None, "cpu") == 2.5
    assert bench.aggregate_rate(1, 100, 4, 2.0) == 200.0
