"""Host side of the uneven work list: the synthetic job mix (no GPU)."""

from __future__ import annotations

import numpy as np


def test_uneven_jobs_shapes_and_ranges(oracle_engine):
    from vfhe_b200.worklist import uneven_jobs

    jobs = uneven_jobs(oracle_engine, count=40, seed=11, logn=(10, 12), limbs=(2, 5), device="cpu")
    kinds = [j.kind for j in jobs]
    assert 10 <= kinds.count("chain") <= 30
    for j in jobs:
        assert 1024 <= j.N <= 4096 and 2 <= j.L <= 5
        assert j.ring.split_degree == 4  # the default split for 50-bit primes
        assert len(j.limbs) == j.L
        qs = np.array(j.ring.primes[: j.L + 1], dtype=np.uint64)
        if j.kind == "chain":
            assert tuple(j.a.shape) == (j.L, j.N) and tuple(j.b.shape) == (j.L, j.N)
            a = j.a.numpy().view(np.uint64)
            assert (a < qs[: j.L, None]).all()
        else:
            assert j.special == j.ring.prime_indices[j.L]
            assert tuple(j.ksk.shape) == (j.L, 2, j.L + 1, j.N)
            k = j.ksk.numpy().view(np.uint64)
            assert (k < qs[None, None, :, None]).all()
        assert j.bytes_moved() > 0


def test_uneven_jobs_are_seeded(oracle_engine):
    from vfhe_b200.arith import reset_registries
    from vfhe_b200.worklist import uneven_jobs

    a = uneven_jobs(oracle_engine, count=6, seed=5, logn=(10, 11), limbs=(2, 3), device="cpu")
    reset_registries()
    b = uneven_jobs(oracle_engine, count=6, seed=5, logn=(10, 11), limbs=(2, 3), device="cpu")
    for x, y in zip(a, b):
        assert (x.kind, x.N, x.L) == (y.kind, y.N, y.L)
        assert np.array_equal(x.a.numpy(), y.a.numpy())


def test_job_semantics_oracle_matches_reference(oracle_engine, ref_portable):
    """The two job kinds, recomputed through the oracle and through the reference
    library's own cdef calls, agree bit for bit (pins what the GPU work list must produce)."""
    from tests.helpers import job_on_engine
    from vfhe_b200.arith import reset_registries
    from vfhe_b200.worklist import uneven_jobs

    jobs = uneven_jobs(oracle_engine, count=8, seed=21, logn=(10, 11), limbs=(2, 4), device="cpu")
    assert {j.kind for j in jobs} == {"chain", "keyswitch"}
    for j in jobs:
        reset_registries()
        want = job_on_engine(ref_portable, j)
        reset_registries()
        got = job_on_engine(oracle_engine, j)
        assert np.array_equal(got, want), (j.kind, j.N, j.L)
