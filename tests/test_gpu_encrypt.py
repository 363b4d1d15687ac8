"""Batched RLWE encryption on the GPU (vfhe_cuda_rlwe_encrypt_batch) and the device
ChaCha20 generator (vfhe_cuda_prng_blocks).

Sampling cannot match the reference's random stream, so encryption is checked by what
must hold for every draw: the phase b - a s, computed on the CPU oracle engine, minus
the message is one small integer e per coefficient, the same in every limb; and by
statistics of a (uniform residues) and e (rounded Gaussian of the given width)."""

from __future__ import annotations

import numpy as np
import pytest

from tests.test_prng_host import golden_cases

pytestmark = pytest.mark.gpu


def test_prng_blocks_match_golden(cuda):
    import torch

    ffi, lib = cuda.ffi, cuda.lib
    for case in golden_cases():
        n = len(case["blocks"])
        out = torch.zeros(n * 16, dtype=torch.int32, device="cuda")
        key = ffi.new("uint32_t[8]", case["key_words"])
        rc = lib.vfhe_cuda_prng_blocks(ffi.cast("uint32_t*", out.data_ptr()), n, key, case["counter"],
                                       case["nonce"], ffi.NULL)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32).reshape(n, 16)
        assert np.array_equal(got, np.array(case["blocks"], dtype=np.uint32))


def _scheme(cuda, N, n_mid, split, seed):
    from vfhe_b200.arith import Ring
    from vfhe_b200.fhe import CKKS_Scheme
    from vfhe_b200.native import use_engine

    with use_engine(cuda):
        rng = np.random.default_rng(seed)
        R = Ring(N, prime_size=[50] + [40] * n_mid, split_degree=split)
        s = CKKS_Scheme(R, scaling_factor=2**40, special_primes=0)
        key = s.key_gen_uniform_ternary(3.2, rng)
    return R, s, key, rng


def _noise(oracle_engine, R, key, out, msgs):
    """e = b - a s - m per limb (oracle engine), centred; asserts one integer per coefficient."""
    from tests.helpers import poly_from_rows
    from vfhe_b200.arith import Polynomial, Ring

    Ro = Ring(R.N, prime_size=[50] * R.ell, primes=R.primes, split_degree=R.split_degree, engine=oracle_engine)
    sk = Polynomial(Ro).from_array(key.key[0])
    sk.to_NTT()
    q = np.array(R.primes, dtype=object)[:, None]
    es = []
    for b in range(out.shape[0]):
        a = poly_from_rows(Ro, out[b, 0])
        a.to_NTT()
        prod = a * sk
        prod.to_coeff()
        phase = (out[b, 1].astype(object) - prod.rows().astype(object)) % q
        e = (phase - msgs[b].astype(object)) % q
        e = np.where(e > q // 2, e - q, e).astype(np.int64)
        assert (e == e[0]).all(), "the noise must be the same integer in every limb"
        es.append(e[0])
    return np.stack(es)


@pytest.mark.parametrize("N,n_mid,split", [(2**12, 3, 1), (2**12, 2, 2), (2**13, 1, 4), (2**12, 1, 8), (2**13, 1, 16)])
def test_encryptions_decrypt_to_message_plus_small_noise(cuda, oracle_engine, N, n_mid, split):
    import torch

    from vfhe_b200.batch import CkksBatch, to_device

    R, s, key, rng = _scheme(cuda, N, n_mid, split, seed=3)
    B = 6
    msgs = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in R.primes]) for _ in range(B)])
    out = CkksBatch(R, 0).encrypt(key, to_device(msgs))
    torch.cuda.synchronize()
    e = _noise(oracle_engine, R, key, out.cpu().numpy().view(np.uint64), msgs)
    assert np.abs(e).max() <= 8 * 3.2
    assert abs(e.std() - 3.2) < 0.2
    assert abs(e.mean()) < 0.1


def test_sample_statistics(cuda, oracle_engine):
    import torch

    from vfhe_b200.batch import CkksBatch

    R, s, key, rng = _scheme(cuda, 2**12, 1, 1, seed=9)
    out = CkksBatch(R, 0).encrypt(key, None, batch=48)
    torch.cuda.synchronize()
    host = out.cpu().numpy().view(np.uint64)
    # a: uniform residues, 16 equal buckets per limb (chi-square, 15 degrees of freedom)
    for i, q in enumerate(R.primes):
        buckets = (host[:, 0, i].astype(object) * 16 // q).astype(np.int64).ravel()
        counts = np.bincount(buckets, minlength=16)
        expect = buckets.size / 16
        chi2 = float(((counts - expect) ** 2 / expect).sum())
        assert chi2 < 45.0, chi2  # p ~ 1e-4 at 15 degrees of freedom
    # e: rounded Gaussian of width 3.2 (encryptions of zero)
    e = _noise(oracle_engine, R, key, host[:8], np.zeros((8, R.ell, R.N), dtype=np.uint64))
    assert abs(e.std() - 3.2) < 0.1
    assert abs(e.mean()) < 0.05
    assert abs(float((e == 0).mean()) - 0.1241) < 0.01  # P(round(N(0, 3.2)) = 0)


def test_deterministic_seed_reproduces_and_distinct_seeds_differ(cuda):
    import torch

    from vfhe_b200.batch import CkksBatch

    R, s, key, rng = _scheme(cuda, 2**12, 1, 1, seed=4)
    enc = CkksBatch(R, 0)
    try:
        cuda.lib.vfhe_prng_set_deterministic_seed(77)
        o1 = enc.encrypt(key, None, batch=3).cpu().numpy()
        cuda.lib.vfhe_prng_set_deterministic_seed(77)
        o2 = enc.encrypt(key, None, batch=3).cpu().numpy()
        o3 = enc.encrypt(key, None, batch=3).cpu().numpy()  # the stream moved on
        cuda.lib.vfhe_prng_set_deterministic_seed(78)
        o4 = enc.encrypt(key, None, batch=3).cpu().numpy()
    finally:
        cuda.lib.vfhe_prng_clear_deterministic_seed()
    torch.cuda.synchronize()
    assert np.array_equal(o1, o2)
    assert not np.array_equal(o1, o3)
    assert not np.array_equal(o1, o4)


def test_ckks_round_trip_through_batched_encryption(cuda):
    """encode -> batched encryption -> decrypt and decode through the reference-API
    mirror: the slots come back within the CKKS error."""
    import torch

    from vfhe_b200.arith import repr
    from vfhe_b200.batch import CkksBatch, to_device
    from vfhe_b200.fhe import CKKS_Ciphertext
    from vfhe_b200.native import use_engine

    R, s, key, rng = _scheme(cuda, 2**12, 3, 1, seed=12)
    zs, msgs = [], []
    with use_engine(cuda):
        for _ in range(3):
            z = np.sqrt(rng.random(R.N // 2)) * np.exp(2j * np.pi * rng.random(R.N // 2))
            p = s.encode(list(z))
            p.to_coeff()
            zs.append(z)
            msgs.append(p.rows())
    out = CkksBatch(R, 0).encrypt(key, to_device(np.stack(msgs)))
    torch.cuda.synchronize()
    host = out.cpu().numpy().view(np.uint64)
    with use_engine(cuda):
        for b, z in enumerate(zs):
            ct = CKKS_Ciphertext(s)
            ct.set_component_rows(0, host[b, 0])
            ct.set_component_rows(1, host[b, 1])
            ct.repr = repr.coeff
            dec = np.array(s.decode(s.decrypt(ct, key)))
            assert np.abs(dec - z).max() < 1e-6
