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


def test_gpus_two_starts_two_ranks_itself():
    """`bench.py --gpus 2` without torchrun's environment launches two ranks
    (torch.distributed.run, rendezvous on 127.0.0.1) and the line rank 0
    prints reports both; the host selftest step stands in for the projector."""
    import json
    import subprocess
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--selftest",
                        "--steps", "3", "--warmup", "3"], capture_output=True, text=True, env=env,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2
    assert line["ms_per_step"] >= line["rank_ms"]
    per_rank = 2 * 256 ** 3 / (line["ms_per_step"] * 1e-3) / 1e9
    assert line["value"] == pytest.approx(2 * per_rank)


def test_rank_count_must_match_gpus():
    """A run whose torchrun environment holds fewer ranks than --gpus asks for
    stops instead of reporting a smaller job under the larger name."""
    import subprocess
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--selftest",
                        "--steps", "1"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode != 0
    assert "1 ranks started for --gpus 2" in r.stderr


def test_reference_arm_line_carries_the_shared_config(monkeypatch, capsys):
    """Both arms print the same `config` (bench.run_config) and at least three
    warm-up steps, so the two lines describe one workload; the reference's CPU
    projector is stubbed here (its timing is not under test)."""
    import argparse
    import json
    sys.path.insert(0, ROOT)
    import bench
    seen = {}

    def fake_run(steps, warmup):
        seen.update(steps=steps, warmup=warmup)
        return 4.0, 6.5, {"kind": "reference", "cores": 16, "sample": "stub"}
    monkeypatch.setattr(bench, "cpu_reference_run", fake_run)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    bench.reference_arm(argparse.Namespace(gpus=1, steps=20, warmup=1))
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["config"] == bench.run_config(1)
    assert line["config"]["n"] == 2048 and line["config"]["np"] == 1440
    assert line["steps"] == 20 and line["warmup"] == 3 and seen == {"steps": 20, "warmup": 3}
    assert line["impl"] == "reference" and line["e2e"]["value"] == line["value"]


def test_summary_reads_the_line_layout():
    """bench.summary() on a line of the GPU arm's layout (pass times beside the
    shared config, optional legs absent): the headline figures come out rounded."""
    sys.path.insert(0, ROOT)
    import bench
    line = {"value": 3158.04, "config": bench.run_config(1),
            "pass_ms": {"forward": 3.5721, "backward": 4.5903},
            "e2e": {"value": 2947.2}, "roofline": {"issue": {"frac": 0.6512}, "shared": {"frac": 0.8013}},
            "cpu_baseline": {"value": 3.87}}
    out = bench.summary(line)
    assert out["fwd_ms"] == 3.572 and out["bwd_ms"] == 4.59 and out["gray_px_s"] == 3158.0
    assert out["e2e_gray_px_s"] == 2947.0 and out["issue_frac"] == 0.651 and out["shared_frac"] == 0.801
    assert out["cpu_gray_px_s"] == 3.87 and "bhc_fan_2048" not in out
