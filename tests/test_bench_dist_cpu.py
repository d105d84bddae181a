"""The multi-GPU host logic of bench.py on CPU (gloo, two ranks): replicas only, so the
only collectives are the barrier and the max-over-ranks of the timed region; the
whole-job rate is every rank's units over the slowest rank's time; the reference arm runs
on rank 0 alone."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(dist, 10.0 + 5.0 * rank, "cpu")   # rank 1 is the slower one
        dist.barrier()
        out[rank] = (ms, bench.whole_job_rate(world, 1000, ms))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_with_two_gloo_ranks():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    assert out[0] == out[1] == (15.0, 2 * 1000 / 15e-3)


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(None, 7.5, "cpu") == 7.5
    assert bench.whole_job_rate(1, 3000, 1.5) == pytest.approx(2e6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    args = bench.argparse.Namespace(scale=1.0, steps=3, warmup=3, ref_budget=1.0)
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""


def test_reference_arm_line_matches_ours_without_the_reference_build(monkeypatch, capsys, tmp_path):
    """Where oracle/_ref holds no reference build the arm falls back to the host port and
    says so; its config carries the same keys as our arm's."""
    import json
    monkeypatch.setenv("WORLD_SIZE", "1")
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setattr(bench, "harness_path", lambda: str(tmp_path / "absent"))
    args = bench.argparse.Namespace(scale=1.0 / 256, steps=1, warmup=0, ref_budget=5.0, gpus=1, no_batch=True)
    assert bench.run_reference(args) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["cpu_baseline"]["kind"] == "port"
    assert "absent" in line["cpu_baseline"]["sample"]
    assert set(line["config"]) == set(bench.bench_config(bench.make_spec(1.0), 1))
    assert line["e2e"]["value"] == line["value"]


def test_every_kth_spreads_the_sample():
    assert bench.every_kth(list(range(64)), 16) == list(range(0, 64, 4))
    assert bench.every_kth([1, 2, 3], 8) == [1, 2, 3]
