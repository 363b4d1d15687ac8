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
    """A work-list job recomputed through the cdef surface of `engine` (reference API):
    chain  = polynomial_RNSc_to_RNS of both operands, polynomial_mul_RNS_polynomial,
             polynomial_RNS_to_RNSc;
    keyswitch = mlwe_RNSc_GHS_hybrid_keyswitch of the rank-1 sample with one key."""
    from vfhe_b200.mlwe import MLWE, MLWE_Scheme, MLWE_Set

    host = lambda t: t.cpu().numpy().view(np.uint64)  # noqa: E731
    L = job.L
    if job.kind == "chain":
        R = Ring(job.N, prime_size=[50] * L, primes=job.ring.primes[:L], split_degree=job.ring.split_degree,
                 engine=engine)
        a = poly_from_rows(R, host(job.a))
        b = poly_from_rows(R, host(job.b))
        c = a * b
        c.to_coeff()
        return c.rows()
    R = Ring(job.N, prime_size=[50] * (L + 1), primes=job.ring.primes[: L + 1], split_degree=job.ring.split_degree,
             engine=engine)
    s = MLWE_Scheme(R, special_primes=1, module_rank=1, max_lvl=1)
    ct, ksk = host(job.a), host(job.ksk)
    c = MLWE(s)
    c.set_component_rows(0, ct[0])
    c.set_component_rows(1, ct[1])
    c.repr = repr.coeff
    comps = []
    for j in range(L):
        k = MLWE(s, ring=s.special_rings[0])
        k.set_component_rows(0, ksk[j][0])
        k.set_component_rows(1, ksk[j][1])
        k.repr = repr.ntt
        comps.append(k)
    out = s.keyswitch(c, MLWE_Set([comps]))
    return np.stack([out.component_rows(0), out.component_rows(1)])
