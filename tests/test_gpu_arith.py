"""cuda engine vs the CPU oracle, bit for bit, on the arith surface (§8 rows a1-a7, a11, a13).

Every case builds the same ring on both engines, injects identical seeded residues,
runs one entry point on each and compares the raw rows (and masks).
"""

from __future__ import annotations

import numpy as np
import pytest

from vfhe_b200.arith import Polynomial, repr

from .helpers import poly_from_rows, same, twin_rings, uniform_rows

pytestmark = pytest.mark.gpu

RINGS = [
    (16, [50, 50], 1),
    (256, [50, 50, 50], None),      # default split 4, as in the reference's tests
    (1024, [20, 20], 8),
    (4096, [50, 50, 50], None),     # config 0, split 4 (P = 1024)
    (4096, [50, 50, 50], 1),        # config 0, split 1
    (2**14, [50] + [40] * 8 + [50], 1),  # CKKS config
    (2**15, [50, 50], 1),           # two-pass transform
    (2**16, [50, 50], 1),           # two-pass transform, N = 2^16
    (2**16, [50, 50], 4),
]


@pytest.fixture
def engines(cuda, oracle_engine):
    """[engine under test, checker]"""
    return [cuda, oracle_engine]


@pytest.fixture(params=RINGS, ids=lambda p: f"N{p[0]}-s{p[2]}-L{len(p[1])}")
def rings(request, engines):
    N, sizes, split = request.param
    return twin_rings(engines, N, sizes, split)


def pair(rings, rng, rep=repr.coeff):
    rows = uniform_rows(rings[0], rng)
    return poly_from_rows(rings[0], rows, rep), poly_from_rows(rings[1], rows, rep)


def test_forward_inverse(rings):
    rng = np.random.default_rng(1)
    g, o = pair(rings, rng)
    g.to_NTT()
    o.to_NTT()
    same(g, o)
    g.to_coeff()
    o.to_coeff()
    same(g, o)


@pytest.mark.parametrize("bits", [30, 40, 45, 49, 50])
@pytest.mark.parametrize("logn", [8, 10, 12, 13, 14, 15, 16, 17])
def test_transform_prime_sizes_and_extremes(engines, bits, logn):
    """Every transform schedule (one tile, column + tile) and both butterfly arithmetics
    at the edges of their ranges: primes just below 2^bits and residues at 0 and q-1."""
    rings = twin_rings(engines, 1 << logn, [bits], 1)
    q = rings[0].primes[0]
    rng = np.random.default_rng(logn * 100 + bits)
    N = 1 << logn
    cases = [
        np.full((1, N), q - 1, dtype=np.uint64),
        np.tile(np.array([0, q - 1], dtype=np.uint64), N // 2)[None, :],
        rng.integers(0, q, (1, N), dtype=np.uint64),
    ]
    for rows in cases:
        g, o = poly_from_rows(rings[0], rows), poly_from_rows(rings[1], rows)
        g.to_NTT()
        o.to_NTT()
        same(g, o)
        g2, o2 = poly_from_rows(rings[0], rows, repr.ntt), poly_from_rows(rings[1], rows, repr.ntt)
        g2.to_coeff()
        o2.to_coeff()
        same(g2, o2)


def test_round_trip_identity(rings):
    rng = np.random.default_rng(2)
    rows = uniform_rows(rings[0], rng)
    g = poly_from_rows(rings[0], rows)
    g.to_NTT()
    g.to_coeff()
    assert np.array_equal(g.rows(), rows)


@pytest.mark.parametrize("op", ["mul", "multo", "add", "sub", "neg", "scale", "scale_rns", "add_int_ntt",
                                "add_int_coeff", "eq"])
def test_elementwise(rings, op):
    rng = np.random.default_rng(3)
    g1, o1 = pair(rings, rng, repr.ntt)
    g2, o2 = pair(rings, rng, repr.ntt)
    scalars = [int(x) for x in rng.integers(1, 2**40, g1.ring.ell)]
    results = []
    for a, b in ((g1, g2), (o1, o2)):
        if op == "mul":
            r = a * b
        elif op == "multo":
            a *= b
            r = a
        elif op == "add":
            r = a + b
        elif op == "sub":
            r = a - b
        elif op == "neg":
            r = -a
        elif op == "scale":
            r = a * 123456789123
        elif op == "scale_rns":
            r = a * scalars
        elif op == "add_int_ntt":
            r = a + (-987654321)
        elif op == "add_int_coeff":
            a.repr = repr.coeff
            r = a + 987654321
        else:
            c = a.copy()
            assert a == c
            c.row(c.ring.prime_indices[0])[5] ^= np.uint64(1)
            assert not (a == c)
            r = a
        results.append(r)
    same(*results)


@pytest.mark.parametrize("gen_pow", [1, 3, 7])
def test_permute(rings, gen_pow):
    rng = np.random.default_rng(4)
    g, o = pair(rings, rng)
    N = rings[0].N
    gen = pow(5, gen_pow, 2 * N)
    same(g.automorphism(gen), o.automorphism(gen))
    same(g.automorphism(2 * N - 1), o.automorphism(2 * N - 1))


def test_mod_reduce_lifted_and_division(rings):
    rng = np.random.default_rng(5)
    g, o = pair(rings, rng)
    if rings[0].ell < 2:
        pytest.skip("needs two limbs")
    q_last = rings[0].primes[-1]
    same(g % q_last, o % q_last)
    sub = [r.quotient_ring(ell=r.ell - 1) for r in rings]
    g2, o2 = g.copy(), o.copy()
    g.round_division(sub[0])
    o.round_division(sub[1])
    same(g, o)
    g2.floor_division(sub[0])
    o2.floor_division(sub[1])
    same(g2, o2)


def test_scaled_lift_and_base_extension(rings):
    if rings[0].ell < 3:
        pytest.skip("needs three limbs")
    rng = np.random.default_rng(6)
    subs = [r.quotient_ring(ell=2) for r in rings]
    rows = uniform_rows(subs[0], rng)
    g = poly_from_rows(subs[0], rows)
    o = poly_from_rows(subs[1], rows)
    same(g.scaled_lift(rings[0]), o.scaled_lift(rings[1]))
    same(g.base_extend(rings[0]), o.base_extend(rings[1]))


def test_mul_by_xai(engines):
    from vfhe_b200.mlwe import MLWE, MLWE_Scheme

    rings = twin_rings(engines, 1024, [50, 50, 50], 1)
    schemes = [MLWE_Scheme(R) for R in rings]
    rng = np.random.default_rng(7)
    for a in (0, 1, 5, 8, 1023, 1024, 1500, 2047, 4096 + 3):
        rows = [uniform_rows(schemes[0].ring, rng) for _ in range(2)]
        res = []
        for s in schemes:
            c = MLWE(s)
            for comp in range(2):
                c.set_component_rows(comp, rows[comp])
            c.repr = repr.coeff
            res.append((c.mul_by_xai(a), c.mul_by_xai(a, minus1=True)))
        for k in range(2):
            for comp in range(2):
                same(res[0][k].component(comp), res[1][k].component(comp))


def test_slots_and_inverse(engines, ref_portable):
    # slot ops and inversion are checked against the reference library directly
    rings = twin_rings([engines[0], ref_portable], 256, [50, 50], 1)
    rng = np.random.default_rng(8)
    rows = uniform_rows(rings[0], rng)
    rows[rows == 0] = 1
    g = poly_from_rows(rings[0], rows, repr.ntt)
    r = poly_from_rows(rings[1], rows, repr.ntt)
    same(g.fast_inverse(), r.fast_inverse())
    outs = []
    for p in (g, r):
        lib, R = p.ring.lib, p.ring
        b = Polynomial(R)
        lib.polynomial_RNS_broadcast_slot(b.obj, p.obj, 7)
        rot = Polynomial(R)
        lib.polynomial_RNS_rotate_slot(rot.obj, p.obj, 9)
        cp = p.copy()
        lib.polynomial_RNS_copy_slot(cp.obj, 3, p.obj, 11)
        outs.append((b, rot, cp))
    for x, y in zip(*outs):
        same(x, y)
