"""Batches larger than one pass of the CKKS kernels takes (their grids' y dimension,
at most 65535, counts up to batch x 2 x (nlimbs + 1) rows): the batched multiply,
rotation and key switch run them as consecutive chunks, and every ciphertext's result
equals the one a call on a smaller batch holding it gives (bit for bit).  Residues are
uniform in [0, q) per limb: the arithmetic is exact, so random rows test it as well as
encryptions would."""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu

N, L = 1024, 3  # one 50-bit and two 40-bit primes + a 50-bit special prime


def _uniform(shape, primes, axis, gen):
    import torch

    t = torch.empty(shape, dtype=torch.int64, device="cuda")
    for k, q in enumerate(primes):
        sl = [slice(None)] * len(shape)
        sl[axis] = k
        t[tuple(sl)].random_(0, q, generator=gen)
    return t


@pytest.fixture(scope="module")
def setup(cuda):
    import torch

    from vfhe_b200.arith import Ring
    from vfhe_b200.fhe import CKKS_Scheme
    from vfhe_b200.native import use_engine

    with use_engine(cuda):
        R = Ring(N, prime_size=[50, 40, 40, 50], split_degree=1)
        s = CKKS_Scheme(R, scaling_factor=2**40, special_primes=1)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(11)
    ext = s.special_rings[0].primes
    chunk = 65535 // (2 * (L + 1))  # the entry points' chunk for L limbs
    B = 16400  # three multiply chunks (the last ragged); the rotation below at L - 1 = 2
    # limbs permutes 2 x 2 x 16400 = 65600 rows, past one grid's 65535
    ct1 = _uniform((B, 2, L, N), s.rings[0].primes, 2, gen)
    ct2 = _uniform((B, 2, L, N), s.rings[0].primes, 2, gen)
    rlk = _uniform((L, 2, L + 1, N), ext, 2, gen)
    return s, ct1, ct2, rlk, chunk, B


def test_multiply_and_rotate_past_one_chunk(cuda, setup):
    import torch

    from vfhe_b200.batch import CkksBatch

    s, ct1, ct2, rlk, chunk, B = setup
    special = s.special_rings[0].prime_indices[-1]
    mul = CkksBatch(s.rings[0], special)
    out = mul.mul_relin_rescale(ct1, ct2, rlk)
    torch.cuda.synchronize()
    assert out.shape[0] == B
    for lo, hi in ((0, 20), (chunk - 10, chunk + 10), (B - 20, B)):
        part = CkksBatch(s.rings[0], special).mul_relin_rescale(ct1[lo:hi].contiguous(), ct2[lo:hi].contiguous(), rlk)
        torch.cuda.synchronize()
        assert torch.equal(part, out[lo:hi]), (lo, hi)

    # the rotation at L - 1 limbs: two passes of at most 65535 // (2 L) ciphertexts
    gk = rlk[: L - 1, :, [0, 1, 3]].contiguous()  # key-shaped: the rotation's L - 1 limbs + the special prime
    rot = CkksBatch(s.rings[1], special)
    big = out
    assert 2 * (L - 1) * big.shape[0] > 65535
    gens = [5] * big.shape[0]
    r = rot.rotate(big.contiguous(), gens, [gk] * big.shape[0])
    torch.cuda.synchronize()
    n = big.shape[0]
    for lo, hi in ((0, 16), (65535 // (2 * L) - 8, 65535 // (2 * L) + 8), (n - 16, n)):
        part = CkksBatch(s.rings[1], special).rotate(big[lo:hi].contiguous(), gens[lo:hi], [gk] * (hi - lo))
        torch.cuda.synchronize()
        assert torch.equal(part, r[lo:hi]), (lo, hi)
    assert cuda.lib.vfhe_cuda_status() == 0
    assert cuda.lib.vfhe_cuda_device_faults() == 0
