"""bench.py's multi-rank plumbing on CPU: two gloo ranks (the GPU run uses
NCCL with the same calls).  The job's time is the slowest rank's, and the
whole-job GLUPS counts every rank's replica; the reference arm prints on
rank 0 only."""
from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import sys
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        q.put((rank, ms, bench.whole_job_glups(1000, 10, world, ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, glups in res:
        assert ms == 15.0                       # the slowest rank's time on every rank
        assert abs(glups - 1000 * 10 * 2 / 0.015 / 1e9) < 1e-15


def test_single_process_is_unchanged():
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.whole_job_glups(4, 5, 1, 2.0) == 4 * 5 / 0.002 / 1e9


def test_reference_arm_prints_on_rank0_only(capsys, monkeypatch):
    import argparse
    import bench
    monkeypatch.setenv("RANK", "1")
    bench.run_reference(argparse.Namespace(steps=1, gpus=2, workload="cavity256_ra1e5"), {}, {})
    assert capsys.readouterr().out == ""
