"""CKKS rational rescale for non-nested level chains (reference ckks.py:150-202):
scaled lift into the union of both levels' primes, then round division.

The reference's own scenarios (test_ckks.py:137-189: levels sharing two primes, and
disjoint levels) decode within its tolerance on the cuda engine, and the rescaled
residues equal the reference library's for the same ciphertext, bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 256


def _subring(Rq, *indices):
    return Rq.quotient_ring(mask=sum(1 << Rq.prime_indices[i] for i in indices))


def _scheme(engine, sizes, chain, special_chain):
    from vfhe_b200.arith import Ring
    from vfhe_b200.fhe import CKKS_Scheme
    from vfhe_b200.native import use_engine

    with use_engine(engine):
        Rq = Ring(N, split_degree=1, prime_size=sizes)
        rings = [_subring(Rq, *c) for c in chain]
        special = [_subring(Rq, *c) for c in special_chain]
        return CKKS_Scheme(rings, scaling_factor=2**50, special_primes=1, special_rings=special)


CASES = {
    "shared_primes": ([50, 50, 50, 30, 50], [(0, 1, 2), (0, 1, 3)], [(0, 1, 2, 4), (0, 1, 3, 4)]),
    "disjoint_primes": ([40, 40, 51, 58, 50], [(2, 3), (0, 1), (2,)], [(2, 3, 4), (0, 1, 4), (2, 4)]),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_rational_rescale_decodes(cuda, case):
    from vfhe_b200.native import use_engine

    rng = np.random.default_rng(61)
    s = _scheme(cuda, *CASES[case])
    with use_engine(cuda):
        key = s.key_gen_sparse(N // 8, 3.2, rng=rng)
        values = [complex(int(a), int(b)) for a, b in rng.integers(-2, 3, (N // 2, 2))]
        ct = s.encrypt(s.encode(values), key)
        assert ct.lvl == 0
        out = s.rational_rescale(ct)
        assert out.lvl == 1
        dec = s.decode(s.decrypt(out, key), scaling_factor=out.delta)
    assert max(abs(v - d) for v, d in zip(values, dec)) < 0.05


@pytest.mark.parametrize("case", sorted(CASES))
def test_rational_rescale_matches_reference_library(cuda, ref_portable, case):
    from vfhe_b200.arith import repr
    from vfhe_b200.fhe import CKKS_Ciphertext
    from vfhe_b200.native import use_engine

    rng = np.random.default_rng(62)
    outs = []
    rows = None
    for eng in (cuda, ref_portable):
        from vfhe_b200.arith import reset_registries

        reset_registries()
        s = _scheme(eng, *CASES[case])
        with use_engine(eng):
            if rows is None:
                rows = [np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in s.rings[0].primes]) for _ in range(2)]
            ct = CKKS_Ciphertext(s, lvl=0)
            ct.set_component_rows(0, rows[0])
            ct.set_component_rows(1, rows[1])
            ct.repr = repr.coeff
            out = s.rational_rescale(ct)
            out.to_coeff()
            outs.append((np.stack([out.component_rows(0), out.component_rows(1)]), out.delta))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1]
