"""The benchmark's multi-rank logic (barrier-free max-over-ranks timing and whole-job
rate) on two gloo ranks over CPU, as bench.py runs it over NCCL with one rank per GPU."""

from __future__ import annotations

import os
import socket

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    local_ms = [12.5, 20.0][rank]
    ms = bench.max_over_ranks(local_ms, dist, "cpu")
    value = bench.whole_job_rate(256, world, ms)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, value))


def test_max_over_ranks_and_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms, value in res:
        assert ms == 20.0  # both ranks report the slowest rank's time
        assert abs(value - 2 * 256 / 0.020) < 1e-6


def test_single_rank_passthrough():
    import bench

    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.whole_job_rate(256, 1, 10.0) == 25600.0
