"""Test helpers: the same ring on several engines, seeded inputs, row comparison."""

from __future__ import annotations

import numpy as np

from vfhe_b200.arith import Polynomial, Ring, repr


def twin_rings(engines, N, prime_size, split=None, primes=None):
    """One Ring per engine with identical primes and pool layout."""
    first = Ring(N, prime_size=prime_size, split_degree=split, primes=primes, engine=engines[0])
    rings = [first]
    for e in engines[1:]:
        rings.append(Ring(N, prime_size=prime_size, split_degree=first.split_degree, primes=first.primes, engine=e))
    return rings


def uniform_rows(ring: Ring, rng: np.random.Generator) -> np.ndarray:
    return np.stack([rng.integers(0, q, ring.N, dtype=np.uint64) for q in ring.primes])


def poly_from_rows(ring: Ring, rows: np.ndarray, rep=repr.coeff) -> Polynomial:
    p = Polynomial(ring)
    p.set_rows(rows)
    p.rns_mask = ring.mask
    p.repr = rep
    return p


def same(p1: Polynomial, p2: Polynomial, rows_only: bool = False) -> None:
    """Bit-exact comparison of active rows and masks."""
    if not rows_only:
        assert p1.rns_mask == p2.rns_mask, (hex(p1.rns_mask), hex(p2.rns_mask))
    for k, idx in enumerate(p1.ring.prime_indices):
        if (p1.rns_mask >> idx) & 1:
            a, b = p1.row(idx), p2.row(p2.ring.prime_indices[k])
            if not np.array_equal(a, b):
                bad = np.nonzero(a != b)[0]
                raise AssertionError(f"limb {k}: {bad.size} residues differ, first at {bad[0]}: {a[bad[0]]} != {b[bad[0]]}")


def job_on_engine(engine, job) -> np.ndarray:
    """A work-list job recomputed through the cdef surface of `engine`
    (vfhe_b200.worklist.run_job_on_engine)."""
    from vfhe_b200.worklist import run_job_on_engine

    return run_job_on_engine(engine, job)
