"""The multi-GPU path of bench.py is replicas: one independent scene per
rank, no collective on the data path, and the whole-job throughput from the
slowest rank's time (an all-reduce of the times).  Checked here with two
gloo ranks on the CPU: every rank gets the same slowest time and the same
whole-job value, and a barrier lets no rank run ahead."""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        w, r, local = bench.dist_setup(None)
        assert (w, r, local) == (world, rank, rank)
        bench.barrier(world)
        secs, value = bench.replica_throughput(200_000, 1000, world, 1.0 + rank, "gloo")
        out[rank] = (secs, value)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world, port = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert out[0] == out[1]
    secs, value = out[0]
    assert secs == 2.0
    assert value == 200_000 * 1000 * world / 2.0


def test_one_rank_needs_no_process_group():
    import bench
    assert bench.replica_throughput(10, 3, 1, 0.5, None) == (0.5, 60.0)
    bench.barrier(1)
