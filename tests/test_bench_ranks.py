"""bench.py's multi-rank timing on two gloo ranks on the CPU: the job's time
is the slowest rank's, and the throughput counts every rank's cases."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # Rank r took 100 (r + 1) ms of device time for its 16 cases, twice.
        job_ms = bench.max_over_ranks(100.0 * (rank + 1), world, "cpu")
        out.put((rank, job_ms, bench.job_solves_per_s(world, 16, 2, job_ms)))
    finally:
        dist.destroy_process_group()


def test_job_time_is_the_slowest_rank_and_throughput_counts_every_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in results] == [200.0, 200.0]
    # 2 ranks x 16 cases x 2 steps in 0.2 s.
    assert results[0][2] == pytest.approx(2 * 16 * 2 / 0.2)


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
