"""The multi-GPU form of the benchmark is independent replicas (points and pairs do not
interact, src/track.jl:423-443): each rank runs its own pair and the job's time is the slowest
rank's. These run the N > 1 logic as world-size-2 gloo process groups on the CPU."""

import multiprocessing as mp
import os
import socket
import sys
from datetime import timedelta
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench

        # Rank r took 100 * (r + 1) ms for 10 steps of 1000 points.
        ms, rate = bench.replicas_rate(dist, 100.0 * (rank + 1), 1000, 10)
        q.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_replicas_rate_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate in out:
        assert ms == 200.0  # the slowest rank's time, on every rank
        assert rate == pytest.approx(2 * 1000 * 10 / 0.2)  # both ranks' points over it


def test_single_process_rate():
    sys.path.insert(0, str(ROOT))
    import bench

    ms, rate = bench.replicas_rate(None, 50.0, 2000, 5)
    assert ms == 50.0 and rate == pytest.approx(2000 * 5 / 0.05)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    bench.reference_arm(None)  # returns before any work on ranks other than 0
    assert capsys.readouterr().out == ""
