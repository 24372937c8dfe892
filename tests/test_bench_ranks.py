"""The multi-rank plumbing of bench.py on CPU: two `gloo` ranks, launched the
way torchrun would (RANK / WORLD_SIZE / MASTER_ADDR=127.0.0.1), each time its
own copy of the workload; the reported time is the slowest rank's, the job
rate counts every rank's units, the reference arm runs on rank 0 only, and the
CPU baseline and single-GPU extras run only in a one-rank job."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        ms = bench.max_over_ranks(times[rank], dist, "cpu")
        out[rank] = (ms, bench.whole_job_rate(world, 40, ms))
    finally:
        dist.destroy_process_group()


def test_slowest_rank_sets_the_time_and_rate():
    world, port = 2, _free_port()
    times = [80.0, 95.5]
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, port, times, out), nprocs=world, join=True)
    for r in range(world):
        ms, rate = out[r]
        assert ms == 95.5
        assert rate == pytest.approx(world * 40 / 0.0955)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    assert bench.run_reference(None) is None   # returns before touching the arguments
    assert capsys.readouterr().out == ""


def test_cpu_baseline_and_extras_only_in_a_one_rank_job():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.single_gpu_extras(0, 1)
    assert not bench.single_gpu_extras(0, 2)
    assert not bench.single_gpu_extras(1, 2)
    assert not bench.single_gpu_extras(3, 8)
