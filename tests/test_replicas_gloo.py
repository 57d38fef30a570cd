"""Multi-GPU form on the CPU: replicas only (one network per rank, no data
exchange).  Two gloo ranks check the bench's max-over-ranks timing and the
whole-job value, and that the reference arm runs on rank 0 alone."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        my_ms = 100.0 + 25.0 * rank  # the ranks finish at different times
        mx = bench.max_over_ranks(my_ms, world, torch.device("cpu"))
        value = bench.replica_value(world, 1_000_000 * 100 * 10, mx)
        dist.barrier()
        out.put((rank, mx, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_value():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect_ms = 125.0
    for rank, mx, value in res:
        assert mx == expect_ms
        assert value == pytest.approx(world * 1e9 / (expect_ms / 1e3))


def test_reference_arm_runs_on_rank_zero_only():
    import argparse
    import sys

    sys.path.insert(0, ROOT)
    import bench

    args = argparse.Namespace(neurons=1000, side=1000.0, seed=1, placement="uniform", steps=1, warmup=0, precision="fp64")
    assert bench.run_reference(args, world=2, rank=1) is None
