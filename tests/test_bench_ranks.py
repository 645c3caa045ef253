"""The multi-process host logic of bench.py on CPU: two gloo ranks on
127.0.0.1.  Each rank of `bench.py --gpus N` runs its own replica; the job's
time is the slowest rank's (all-reduce MAX) and the job's throughput counts
every rank's points; the reference arm runs on rank 0 alone."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as tmp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        ms = bench.max_over_ranks(1.5 + rank, world)  # rank 1 is the slower one
        e2e = bench.max_over_ranks(10.0 - rank, world)  # rank 0 is the slower one
        value = bench.job_mpts_s(world, 245760, ms)

        class A:
            warmup, steps = 1, 1

        # the reference arm: every rank but 0 returns without work
        if rank != 0:
            bench.run_reference(A(), rank, world)
        out[rank] = (ms, e2e, value)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world = 2
    mgr = tmp.get_context("spawn").Manager()
    out = mgr.dict()
    tmp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert set(out.keys()) == {0, 1}
    for r in range(world):
        ms, e2e, value = out[r]
        assert ms == 2.5 and e2e == 10.0
        assert value == pytest.approx(2 * 245760 / 2.5e-3 / 1e6)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1) == 3.25
    assert bench.job_mpts_s(1, 1000, 1.0) == pytest.approx(1.0)
