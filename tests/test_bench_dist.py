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


# ---- sharding: each rank's pairs are a disjoint block of one seeded job, and what a
# rank computes on its share equals what one rank computes on the whole job

_SHARD_RING = dict(n=256, prime_sizes=[50, 40, 40, 50], gk_steps=[1, 2, 4])
_SHARD_PAIRS = 2  # per rank


def _step_rows(engine, s, rlk, gks, cts, steps):
    """bench.py's per-pair step (multiply, relinearise, rescale, rotate) on the API mirror."""
    import numpy as np

    from vfhe_b200.batch import ciphertext_rows
    from vfhe_b200.native import use_engine

    out = []
    with use_engine(engine):
        for p, k in enumerate(steps):
            prod = s.multiply(cts[2 * p], cts[2 * p + 1], rlk)
            prod.round_division(lvl=1)
            out.append(ciphertext_rows(s.automorphism(prod, s.galois_gen(k), gks[k])))
    return np.stack(out)


def _shard_rank(rank: int, world: int, port: int, q) -> None:
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    import bench
    from tests.conftest import build_oracle
    from vfhe_b200.native import Engine

    eng = Engine(build_oracle(), "oracle")
    share = bench.pair_share(rank, _SHARD_PAIRS)
    s, key, rlk, gks, steps, zs, cts = bench.build_workload(eng, _SHARD_PAIRS, bench.SEED, first_pair=share.start,
                                                            **_SHARD_RING)
    rows = _step_rows(eng, s, rlk, gks, cts, steps)
    got = [None] * world
    dist.all_gather_object(got, (list(share), steps, rows))
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put(got)


def test_ranks_take_disjoint_shares_of_one_job():
    import numpy as np

    import bench
    from tests.conftest import build_oracle
    from vfhe_b200.native import Engine

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    shares = [g[0] for g in got]
    flat = [i for sh in shares for i in sh]
    assert sorted(flat) == list(range(world * _SHARD_PAIRS))  # disjoint and covering the job
    assert shares == [list(bench.pair_share(r, _SHARD_PAIRS)) for r in range(world)]

    # one rank over the whole job
    eng = Engine(build_oracle(), "oracle")
    s, key, rlk, gks, steps, zs, cts = bench.build_workload(eng, world * _SHARD_PAIRS, bench.SEED, **_SHARD_RING)
    whole = _step_rows(eng, s, rlk, gks, cts, steps)
    assert [k for g in got for k in g[1]] == steps
    assert np.array_equal(np.concatenate([g[2] for g in got]), whole)
