"""bench.py's replica aggregation (`--gpus N`): the timed value is all ranks'
updates over the slowest rank's time, gathered with a MAX all-reduce.  Run
with two gloo ranks on the CPU (the GPU run uses the same helpers over NCCL)."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t_ms = [12.5, 14.0][rank]            # each rank's own step time
        t_max = bench.max_over_ranks(t_ms, dist, "cpu")
        out[rank] = (t_max, bench.replica_value(world, 1.0e9, t_max))
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank_and_the_summed_work():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    for rank in (0, 1):
        t_max, value = res[rank]
        assert t_max == 14.0
        assert value == pytest.approx(2 * 1.0e9 / 14.0e-3 / 1e9)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.replica_value(1, 2.0e9, 1000.0) == pytest.approx(2.0)
