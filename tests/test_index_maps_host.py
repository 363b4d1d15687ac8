"""Index arithmetic of two GPU kernels, restated and checked without a GPU.

* The batched Galois permutation (ckks.cu, k_permute_batch) is written as a gather:
  output coefficient c' takes source coefficient p = c' gen^-1 mod 2N (negated when
  p >= N).  It must equal the reference's scatter (rns_polynomial.c:996-1035: c moves
  to c gen mod 2N) for every split degree.
* The lane-major twiddle copy for transform passes over index bits 2..5 (runtime.cu,
  build_prime; ntt_f64.cu, f_fwd_tw / f_inv_tw with LO = 2) must hand every thread the
  twiddle the bit-reversed table gives it: index P/2^(b+1) + (position >> (b+1)).
"""

from __future__ import annotations

import random

import pytest


def scatter(src, N, ls, gen, q):
    S, P = 1 << ls, N >> ls
    dst = [None] * N
    for pos in range(N):
        i, i2 = divmod(pos, P)
        idx = (i + (i2 << ls)) * gen
        d = (idx & (S - 1)) * P + ((idx & (N - 1)) >> ls)
        dst[d] = (q - src[pos]) % q if idx & N else src[pos]
    return dst


def gather(src, N, ls, gen, q):
    x = gen
    for _ in range(6):  # Newton's iteration for gen^-1 mod 2^64, as the host does
        x = (x * (2 - gen * x)) % (1 << 64)
    ginv = x & (2 * N - 1)
    assert ginv * gen % (2 * N) == 1
    S, P = 1 << ls, N >> ls
    log_p, out = P.bit_length() - 1, []
    for d in range(N):
        cd = (d >> log_p) + ((d & (P - 1)) << ls)
        p = (cd * ginv) & (2 * N - 1)  # 32-bit wraparound keeps these bits when 2N <= 2^31
        c = p & (N - 1)
        v = src[((c & (S - 1)) << log_p) + (c >> ls)]
        out.append((q - v) % q if p >= N else v)
    return out


@pytest.mark.parametrize("N", [8, 64, 1024])
def test_permutation_gather_equals_scatter(N):
    rng = random.Random(N)
    q = 97
    for ls in range(0, min(5, N.bit_length() - 1)):
        for gen in {1, 3, 5, 25, 2 * N - 1, rng.randrange(1, 2 * N, 2)}:
            src = [rng.randrange(q) for _ in range(N)]
            assert scatter(src, N, ls, gen, q) == gather(src, N, ls, gen, q), (N, ls, gen)


def own(lo, t, m):
    return ((t >> lo) << (lo + 4)) | (m << lo) | (t & ((1 << lo) - 1))


def lane_index(g, b, h):
    return (((g >> 5) * 15 + ((1 << (3 - b)) - 1) + h) << 5) + (g & 31)


@pytest.mark.parametrize("logP,K", [(14, 10), (10, 10), (15, 10), (13, 10), (8, 6)])
def test_mid_pass_twiddle_copy(logP, K):
    P, tpt = 1 << logP, 1 << (K - 4)
    table = {}
    for g in range(P // 64):
        for bb in range(4):
            for h in range(1 << (3 - bb)):
                table[lane_index(g, bb, h)] = (P >> (bb + 3)) + (g << (3 - bb)) + h
    for hi in range(P >> K):
        for t in range(tpt):
            for b in range(2, 6):
                bb = b - 2
                for h in range(1 << (3 - bb)):
                    direct = (P >> (b + 1)) + (hi << (K - b - 1)) + (own(2, t, h << (bb + 1)) >> (b + 1))
                    g = (hi << (K - 6)) + (t >> 2)
                    assert table[lane_index(g, bb, h)] == direct
