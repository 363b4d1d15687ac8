"""Uneven work list (vfhe_cuda_worklist_*): every job bit-exact with the one-call path
and with the oracle engine (reference API: polynomial_RNSc_to_RNS / product /
polynomial_RNS_to_RNSc, and mlwe_RNSc_GHS_hybrid_keyswitch); transform schedules
never change results."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", [0, 1], ids=["persistent", "graph"])
@pytest.mark.parametrize("count,logn,limbs,seed", [(24, (10, 13), (2, 6), 5), (6, (14, 16), (2, 3), 6),
                                                   (40, (10, 16), (2, 5), 9)])
def test_worklist_matches_per_call_and_oracle(cuda, oracle_engine, count, logn, limbs, seed, mode):
    import torch

    from tests.helpers import job_on_engine
    from vfhe_b200.worklist import WorkList, per_call_workspace, run_per_call, uneven_jobs

    jobs = uneven_jobs(cuda, count=count, seed=seed, logn=logn, limbs=limbs)
    assert {j.kind for j in jobs} == {"chain", "keyswitch"}
    wl = WorkList(cuda, mode=mode)
    for j in jobs:
        wl.add(j)
    wl.run()
    torch.cuda.synchronize()
    first = [j.out.clone() for j in jobs]
    wl.run()  # a second run (the persistent kernel's barriers start from zero again)
    torch.cuda.synchronize()
    assert all(torch.equal(f, j.out) for f, j in zip(first, jobs))
    if mode == 0:
        assert wl.persistent and wl.launches == 3
    else:
        assert not wl.persistent and wl.launches > 1
    assert cuda.lib.vfhe_cuda_device_faults() == 0

    outs = [torch.empty_like(j.out) for j in jobs]
    run_per_call(cuda, jobs, outs, per_call_workspace(cuda, jobs))
    torch.cuda.synchronize()
    for j, o in zip(jobs, outs):
        assert torch.equal(j.out, o), (j.kind, j.N, j.L)

    # the oracle on a few jobs of each kind
    checked = {"chain": 0, "keyswitch": 0}
    for j in jobs:
        if checked[j.kind] >= 2:
            continue
        want = job_on_engine(oracle_engine, j)
        assert np.array_equal(j.out.cpu().numpy().view(np.uint64), want), (j.kind, j.N, j.L)
        checked[j.kind] += 1
    wl.close()


def test_schedules_do_not_change_results(cuda):
    import torch

    from vfhe_b200.arith import Ring
    from vfhe_b200.batch import to_device, to_host

    ffi, lib = cuda.ffi, cuda.lib
    rng = np.random.default_rng(7)
    st = ffi.cast("void*", torch.cuda.current_stream().cuda_stream)
    # ctas_per_sm = -1: the fused column + tile transform on a thread-block cluster
    cases = [(2**10, 1, [(0, 2, 0), (0, 1, 2), (0, 4, 1), (0, 8, 0)]),
             (2**13, 1, [(0, 1, 0), (11, 0, 0), (12, 1, 2), (12, 0, -1), (11, 0, -1)]),
             (2**14, 1, [(13, 0, 0), (11, 2, 0), (12, 1, 1), (12, 0, -1), (11, 0, -1), (13, 0, -1)]),
             (2**15, 1, [(12, 0, -1), (13, 0, -1)]),
             (2**16, 1, [(13, 0, 0), (12, 0, 2), (11, 4, 0), (11, 2, 0), (13, 0, -1)]),
             (2**16, 4, [(13, 0, 1), (11, 2, 0), (12, 0, -1)])]
    for N, split, scheds in cases:
        R = Ring(N, prime_size=[50] * 3, split_degree=split, engine=cuda)
        logP = (N // split).bit_length() - 1
        B = 2
        rows = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in R.primes]) for _ in range(B)])
        limbs = ffi.new("uint32_t[]", R.prime_indices)

        def fwd_inv():
            x = to_device(rows)
            p = ffi.cast("uint64_t*", x.data_ptr())
            assert lib.vfhe_cuda_ntt_batch(R.NTT, 0, p, p, B, limbs, 3, st) == 0
            torch.cuda.synchronize()
            f = to_host(x)
            assert lib.vfhe_cuda_ntt_batch(R.NTT, 1, p, p, B, limbs, 3, st) == 0
            torch.cuda.synchronize()
            return f, to_host(x)

        nrows = B * 3 * split
        bucket = nrows.bit_length() - 1
        base_f, base_i = fwd_inv()
        assert np.array_equal(base_i, rows)
        for tb, tpc, cps in scheds:
            assert lib.vfhe_cuda_ntt_set_schedule(logP, bucket, tb, tpc, cps) == 0
            got = ffi.new("int32_t[3]")
            lib.vfhe_cuda_ntt_get_schedule(logP, nrows, got)
            assert list(got) == [tb, tpc, cps]
            f, i = fwd_inv()
            assert np.array_equal(f, base_f), (N, split, tb, tpc, cps)
            assert np.array_equal(i, rows), (N, split, tb, tpc, cps)
        assert lib.vfhe_cuda_ntt_set_schedule(logP, bucket, 0, 0, 0) == 0
    # shapes outside the supported set are refused
    assert lib.vfhe_cuda_ntt_set_schedule(14, 3, 7, 0, 0) != 0
    lib.vfhe_cuda_clear_error()
    assert lib.vfhe_cuda_device_faults() == 0  # no bounded tile-copy wait gave up


def test_persistent_double_buffered_schedules(cuda):
    """Grids smaller than the tile count take the persistent path (bulk asynchronous
    tile loads into two shared buffers); results must equal the one-CTA-per-tile path."""
    import torch

    from vfhe_b200.arith import Ring
    from vfhe_b200.batch import to_device, to_host

    ffi, lib = cuda.ffi, cuda.lib
    rng = np.random.default_rng(8)
    st = ffi.cast("void*", torch.cuda.current_stream().cuda_stream)
    for N, split, B, scheds in [(2**12, 1, 512, [(12, 0, 1), (12, 0, 2), (11, 2, 1)]),
                                (2**10, 1, 1024, [(10, 4, 1), (10, 2, 2)]),
                                (2**14, 1, 96, [(12, 0, 1), (11, 2, 2), (13, 0, 1)]),
                                (2**16, 4, 24, [(12, 0, 2)])]:
        R = Ring(N, prime_size=[50] * 3, split_degree=split, engine=cuda)
        logP = (N // split).bit_length() - 1
        rows = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in R.primes]) for _ in range(B)])
        limbs = ffi.new("uint32_t[]", R.prime_indices)
        nrows = B * 3 * split
        bucket = nrows.bit_length() - 1

        def fwd_inv():
            x = to_device(rows)
            p = ffi.cast("uint64_t*", x.data_ptr())
            assert lib.vfhe_cuda_ntt_batch(R.NTT, 0, p, p, B, limbs, 3, st) == 0
            f = x.clone()
            assert lib.vfhe_cuda_ntt_batch(R.NTT, 1, p, p, B, limbs, 3, st) == 0
            torch.cuda.synchronize()
            return f, x

        saved = ffi.new("int32_t[3]")
        lib.vfhe_cuda_ntt_get_schedule(logP, nrows, saved)
        assert lib.vfhe_cuda_ntt_set_schedule(logP, bucket, 0, 0, 0) == 0
        base_f, base_i = fwd_inv()
        assert np.array_equal(to_host(base_i), rows)
        for tb, tpc, cps in scheds:
            assert lib.vfhe_cuda_ntt_set_schedule(logP, bucket, tb, tpc, cps) == 0
            f, i = fwd_inv()
            assert torch.equal(f, base_f), (N, split, tb, tpc, cps)
            assert torch.equal(i, base_i), (N, split, tb, tpc, cps)
        assert lib.vfhe_cuda_ntt_set_schedule(logP, bucket, *saved) == 0
    assert lib.vfhe_cuda_device_faults() == 0
