"""The uniform sampler's rejection rule (uniform_mod64 in csrc/chacha.cuh, Lemire's
multiply-shift with rejection): for a w-bit uniform r and m = r q, keeping hi(m) only
when lo(m) >= 2^w mod q gives every residue in [0, q) the same number of accepted r.
Checked exhaustively at small word sizes, where every r can be enumerated, and the
threshold the kernel computes as (0 - q) mod q in 64-bit arithmetic is checked to equal
2^64 mod q for primes of the sizes the engine uses."""

from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("w", [8, 12, 16])
@pytest.mark.parametrize("q", [3, 5, 7, 97, 193, 241, 251])
def test_rejection_rule_is_exactly_uniform(w, q):
    if q >= 1 << w:
        pytest.skip("q must be below 2^w")
    r = np.arange(1 << w, dtype=np.uint64)
    m = r * np.uint64(q)
    hi = m >> np.uint64(w)
    lo = m & np.uint64((1 << w) - 1)
    thresh = (1 << w) % q
    kept = hi[lo >= np.uint64(thresh)]
    counts = np.bincount(kept.astype(np.int64), minlength=q)
    assert counts.size == q  # every output below q
    assert (counts == (1 << w) // q).all()  # and equally often
    assert (1 << w) - kept.size == thresh  # exactly 2^w mod q draws rejected


def test_device_threshold_formula():
    rng = np.random.default_rng(3)
    for bits in (30, 40, 50, 61):
        for _ in range(20):
            q = int(rng.integers(1 << (bits - 1), 1 << bits)) | 1
            assert ((2**64 - q) % 2**64) % q == 2**64 % q
