"""The batched device API must reproduce the one-op-per-call path bit for bit.

Reference path: CKKS_Ciphertext multiply (mlwe_multiply + rescale) and rotate
through the cdef surface; batched path: vfhe_cuda_ckks_mul_relin_rescale_batch and
vfhe_cuda_ckks_rotate_batch over device tensors.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(cuda, N, n_mid, pairs, steps, seed, split=1):
    from vfhe_b200.arith import Ring
    from vfhe_b200.fhe import CKKS_Scheme
    from vfhe_b200.native import use_engine

    with use_engine(cuda):
        rng = np.random.default_rng(seed)
        R = Ring(N, prime_size=[50] + [40] * n_mid + [50], split_degree=split)
        s = CKKS_Scheme(R, scaling_factor=2**40, special_primes=1)
        key = s.key_gen_uniform_ternary(3.2, rng)
        rlk = s.gen_rlk(key, key, lvl=0, rng=rng)
        gks = {k: s.gen_ksk_automorphism(key, key, s.galois_gen(k), lvl=1, rng=rng) for k in steps}
        cts = []
        for _ in range(pairs):
            z = np.sqrt(rng.random(N // 2)) * np.exp(2j * np.pi * rng.random(N // 2))
            cts.append(s.encrypt(s.encode(list(z)), key, rng=rng))
        return s, key, rlk, gks, cts


@pytest.mark.parametrize("N,n_mid,split", [(2**12, 3, 1), (2**14, 8, 1), (2**12, 3, None), (2**13, 2, 2),
                                           (2**8, 2, 1)])
def test_batched_ckks_matches_single_calls(cuda, N, n_mid, split):
    import torch

    from vfhe_b200.batch import CkksBatch, ciphertext_rows, key_tensor, to_device, to_host

    steps = [1, 4]
    s, key, rlk, gks, cts = _setup(cuda, N, n_mid, 6, steps, seed=31, split=split)
    c1, c2 = cts[0::2], cts[1::2]
    rot_steps = [steps[i % len(steps)] for i in range(len(c1))]

    # one op per call
    ref_prod, ref_rot = [], []
    for a, b, k in zip(c1, c2, rot_steps):
        p = s.multiply(a, b, rlk)
        p.round_division(lvl=1)
        ref_prod.append(ciphertext_rows(p))
        ref_rot.append(ciphertext_rows(s.automorphism(p, s.galois_gen(k), gks[k])))

    # batched
    for c in cts:
        c.to_NTT()
    t1 = to_device(np.stack([ciphertext_rows(c) for c in c1]))
    t2 = to_device(np.stack([ciphertext_rows(c) for c in c2]))
    special = s.special_rings[0].prime_indices[-1]
    out = CkksBatch(s.rings[0], special).mul_relin_rescale(t1, t2, key_tensor(rlk))
    torch.cuda.synchronize()
    assert np.array_equal(to_host(out), np.stack(ref_prod))

    keys = {k: key_tensor(v) for k, v in gks.items()}
    rot = CkksBatch(s.rings[1], special).rotate(out, [s.galois_gen(k) for k in rot_steps],
                                                [keys[k] for k in rot_steps])
    torch.cuda.synchronize()
    assert np.array_equal(to_host(rot), np.stack(ref_rot))


def test_batched_rotate_ragged_key_groups(cuda):
    """11 ciphertexts over 5 Galois keys, in an order that interleaves the keys: the
    key-switch MAC takes ciphertexts in groups sharing a key, and groups that straddle
    two keys or run past the batch end must not change a residue."""
    import torch

    from vfhe_b200.batch import CkksBatch, ciphertext_rows, key_tensor, to_device, to_host

    steps = [1, 2, 4, 8, 16]
    s, key, rlk, gks, cts = _setup(cuda, 2**12, 3, 11, steps, seed=7)
    rot_steps = [steps[(3 * i) % len(steps)] for i in range(len(cts))]
    for c in cts:
        c.round_division(lvl=1)
        c.to_coeff()
    rows = np.stack([ciphertext_rows(c) for c in cts])
    ref = [ciphertext_rows(s.automorphism(c, s.galois_gen(k), gks[k])) for c, k in zip(cts, rot_steps)]
    t = to_device(rows)
    keys = {k: key_tensor(v) for k, v in gks.items()}
    special = s.special_rings[0].prime_indices[-1]
    rot = CkksBatch(s.rings[1], special).rotate(t, [s.galois_gen(k) for k in rot_steps], [keys[k] for k in rot_steps])
    torch.cuda.synchronize()
    assert np.array_equal(to_host(rot), np.stack(ref))


def test_batched_ntt_matches_single_calls(cuda):
    import torch

    from vfhe_b200.arith import Polynomial, Ring, repr
    from vfhe_b200.batch import to_device, to_host

    rng = np.random.default_rng(32)
    for N, L, split in [(2**16, 4, 1), (2**12, 3, 4), (2**14, 10, 1)]:
        R = Ring(N, prime_size=[50] * L, split_degree=split, engine=cuda)
        B = 3
        rows = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in R.primes]) for _ in range(B)])
        ref = []
        for b in range(B):
            p = Polynomial(R)
            p.set_rows(rows[b])
            p.rns_mask = R.mask
            p.repr = repr.coeff
            p.to_NTT()
            ref.append(p.rows())
        x = to_device(rows)
        limbs = cuda.ffi.new("uint32_t[]", R.prime_indices)
        ptr = cuda.ffi.cast("uint64_t*", x.data_ptr())
        st = cuda.ffi.cast("void*", torch.cuda.current_stream().cuda_stream)
        assert cuda.lib.vfhe_cuda_ntt_batch(R.NTT, 0, ptr, ptr, B, limbs, L, st) == 0
        torch.cuda.synchronize()
        assert np.array_equal(to_host(x), np.stack(ref))
        assert cuda.lib.vfhe_cuda_ntt_batch(R.NTT, 1, ptr, ptr, B, limbs, L, st) == 0
        torch.cuda.synchronize()
        assert np.array_equal(to_host(x), rows)
