"""The exact FP64 modular product of csrc/fp64mod.cuh, emulated step by step on the host:
every __dmul_rn / __fma_rn / __dadd_rn is the exact rational result rounded once to the
nearest double (CPython's int / int division rounds correctly), so these checks follow
the device arithmetic operation for operation.  They pin the claim the element-wise
kernels rely on: for canonical y, w < q < 2^50 (uncentred multiplier) and the quotient
estimate wq = fl(w fl(1/q)) that the kernels compute, f_mulmod(y, w, wq, q) is congruent
to y w mod q and small enough that f_to_canonical returns (y w) mod q exactly, also
after adding a second product (the tensor kernel's d1) or a canonical residue (the
encryption's noise term)."""

from __future__ import annotations

from fractions import Fraction

import numpy as np
import pytest

M = 6755399441055744.0  # 1.5 * 2^52


def _rn(x: Fraction) -> float:
    return x.numerator / x.denominator  # correctly rounded to nearest, ties to even


def dmul(a: float, b: float) -> float:
    return _rn(Fraction(a) * Fraction(b))


def fma(a: float, b: float, c: float) -> float:
    return _rn(Fraction(a) * Fraction(b) + Fraction(c))


def dadd(a: float, b: float) -> float:
    return _rn(Fraction(a) + Fraction(b))


def f_mulmod(y: float, w: float, wq: float, q: float) -> float:
    h = dmul(y, w)
    lo = fma(y, w, -h)
    n = dadd(fma(y, wq, M), -M)
    r = fma(-n, q, h)
    return dadd(r, lo)


def f_to_canonical(x: float, q: float, qinv: float, qi: int) -> int:
    n = dadd(fma(x, qinv, M), -M)
    c = fma(-n, q, x)
    assert abs(c) < 2.0**51 and c == int(c)
    v = int(c)  # the kernel reads c + 2^51 out of the mantissa of c + M, then subtracts 2^51
    return v + qi if v < 0 else v


def _moduli():
    rng = np.random.default_rng(17)
    qs = [(1 << 50) - 27, (1 << 50) - 1, (1 << 49) + 1, (1 << 40) - 87, (1 << 30) + 3, 12289]
    for bits in (50, 49, 45, 40, 32):
        qs += [int(rng.integers(1 << (bits - 1), 1 << bits)) | 1 for _ in range(3)]
    return qs


def _operands(q: int, rng):
    edge = [0, 1, 2, q // 2, q // 2 + 1, q - 2, q - 1]
    return edge + [int(v) for v in rng.integers(0, q, 24, dtype=np.uint64)]


@pytest.mark.parametrize("q", _moduli())
def test_uncentred_product_is_exact(q):
    rng = np.random.default_rng(q % 1000)
    qd = float(q)
    qinv = 1.0 / qd
    ops = _operands(q, rng)
    for y in ops:
        for w in ops[:12] + ops[-6:]:
            fw = float(w)
            t = f_mulmod(float(y), fw, dmul(fw, qinv), qd)
            assert abs(t) < 0.75 * q + 2, (y, w)
            assert f_to_canonical(t, qd, qinv, q) == y * w % q, (y, w)


@pytest.mark.parametrize("q", [(1 << 50) - 27, (1 << 40) - 87])
def test_sums_of_products_and_residues_stay_exact(q):
    rng = np.random.default_rng(5)
    qd = float(q)
    qinv = 1.0 / qd
    for _ in range(300):
        a1, b1, a2, b2, e = (int(v) for v in rng.integers(0, q, 5, dtype=np.uint64))
        fa1, fb1 = float(a1), float(b1)
        qa1, qb1 = dmul(fa1, qinv), dmul(fb1, qinv)
        d1 = dadd(f_mulmod(float(b2), fa1, qa1, qd), f_mulmod(float(a2), fb1, qb1, qd))
        assert f_to_canonical(d1, qd, qinv, q) == (a1 * b2 + b1 * a2) % q
        t = dadd(f_mulmod(float(a2), fa1, qa1, qd), float(e))
        assert f_to_canonical(t, qd, qinv, q) == (a1 * a2 + e) % q


@pytest.mark.parametrize("q", [(1 << 50) - 27, (1 << 49) + 1, (1 << 40) - 87])
def test_centred_twiddle_with_lazy_input(q):
    """The butterflies' case: a centred twiddle |w| <= q/2 with wq = fl(w / q) (the
    tables' quotient, a correctly rounded division) and a lazily reduced input
    |y| < 2^52 give |t| <= 3q/4 with t = y w mod q."""
    rng = np.random.default_rng(11)
    qd = float(q)
    ws = [0, 1, -1, q // 2, -(q // 2)] + [int(v) - q // 2 for v in rng.integers(0, q, 20, dtype=np.uint64)]
    ys = [0, 1, -1, (1 << 52) - 1, -((1 << 52) - 1)] + [int(v) for v in rng.integers(-(1 << 52) + 1, 1 << 52, 40)]
    for w in ws:
        fw = float(w)
        wq = _rn(Fraction(w, q))
        for y in ys:
            t = f_mulmod(float(y), fw, wq, qd)
            assert t == int(t) and abs(t) <= 0.75 * q, (y, w)
            assert (int(t) - y * w) % q == 0, (y, w)
