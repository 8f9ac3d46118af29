"""The N > 1 path of bench.py on CPU: two gloo ranks (world size 2) reduce the
whole-job rate exactly as the GPU ranks do over NCCL (sum of every rank's
units over the slowest rank's time), and the reference arm runs on rank 0
only."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dev = torch.device("cpu")
        units = [1000.0, 3000.0][rank]
        seconds = [0.5, 2.0][rank]
        out[rank] = (bench.job_rate(dist, dev, units, seconds),
                     bench.over_ranks(dist, dev, seconds, "max"),
                     bench.over_ranks(dist, dev, units, "sum"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_the_job_rate():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            rate, slowest, total = out[r]
            assert slowest == 2.0 and total == 4000.0
            assert rate == pytest.approx(4000.0 / 2.0)


def test_one_process_is_its_own_job():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.job_rate(None, None, 500.0, 0.25) == 2000.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    called = []
    monkeypatch.setattr(bench, "build_native", lambda: called.append("build"))
    assert bench.reference_arm(type("A", (), {"config": "c2"})()) is None
    assert not called
