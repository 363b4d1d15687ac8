"""Integer helpers for ring setup (reference modules/arith/python/src/vfhe/arith/number_theory.py).

``is_prime`` is a deterministic Miller-Rabin for 64-bit integers (fixed witness
sets by size); ``crt`` reconstructs an integer from its residues.
"""

from __future__ import annotations

import math

_SMALL = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)


def is_prime(n: int) -> bool:
    if n < 2:
        return False
    for p in _SMALL:
        if n == p:
            return True
        if n % p == 0:
            return False
    d, r = n - 1, 0
    while d % 2 == 0:
        d //= 2
        r += 1
    # the first twelve primes are a deterministic witness set for n < 3.3e24
    for a in _SMALL:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(r - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def crt(values, moduli) -> int:
    if len(moduli) == 1:
        return int(values[0]) % int(moduli[0])
    M = math.prod(int(m) for m in moduli)
    acc = 0
    for v, m in zip(values, moduli, strict=True):
        n = M // int(m)
        acc += int(v) * n * pow(n, -1, int(m))
    return acc % M
