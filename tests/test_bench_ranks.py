"""The multi-rank host logic of bench.py on CPU: two gloo ranks, as torchrun would start
them.  With N GPUs the bench runs N independent replicas; the job's time is the slowest
rank's (max over ranks) and its throughput counts every rank's units.  The reference arm
runs on rank 0 alone."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, world)  # rank 1 is the slow one
        out[rank] = (ms, bench.job_rate(1_000_000, 4, world, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time_and_the_job_rate():
    world = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        got = dict(out)
    assert got[0][0] == got[1][0] == 15.0
    # 2 ranks x 4 steps x 1e6 units in 15 ms
    assert got[0][1] == pytest.approx(2 * 4 * 1e6 / 15e-3 / 1e6)
    assert got[0][1] == got[1][1]


def test_single_rank_needs_no_process_group():
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_rate(50, 10, 1, 1000.0) == pytest.approx(50 * 10 / 1.0 / 1e6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    args = bench.parse()
    bench.run_reference(args)  # returns before any work on a rank other than 0
    assert capsys.readouterr().out == ""
