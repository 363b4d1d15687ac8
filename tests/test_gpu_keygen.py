"""Key-switching keys generated on the GPU (vfhe_cuda_gen_ksk_batch).

Keys come from a random stream, so they cannot equal the reference's bit for bit.
They are checked by what every draw must satisfy: each digit decrypts (on the CPU
oracle) to its gadget message plus one small noise integer shared by all limbs; and
by use: a GPU relinearisation key and Galois key drive the batched CKKS multiply and
rotation to the right slots."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(cuda, N, n_mid, seed):
    from vfhe_b200.arith import Ring
    from vfhe_b200.fhe import CKKS_Scheme
    from vfhe_b200.native import use_engine

    with use_engine(cuda):
        rng = np.random.default_rng(seed)
        R = Ring(N, prime_size=[50] + [40] * n_mid + [50], split_degree=1)
        s = CKKS_Scheme(R, scaling_factor=2**40, special_primes=1)
        key = s.key_gen_uniform_ternary(3.2, rng)
    return s, key, rng


def test_digits_decrypt_to_gadget_messages(cuda, oracle_engine):
    import torch

    from tests.helpers import poly_from_rows
    from vfhe_b200.arith import Polynomial, Ring
    from vfhe_b200.batch import gen_rlk_batch
    from vfhe_b200.native import use_engine

    s, key, rng = _setup(cuda, 2**12, 3, seed=21)
    with use_engine(cuda):
        rlk = gen_rlk_batch(s, key, lvl=0, engine=cuda)
        torch.cuda.synchronize()
        sring = s.special_rings[0]
        P = sring.modulus_ratio(s.rings[0])
        src = s.quadratic_key_polys(key)[0]
        src = Polynomial(sring).from_bigint_array(src.get_polynomial(signed=True))
        src.to_coeff()
        src_rows = src.rows()
    host = rlk.cpu().numpy().view(np.uint64)
    L, N = sring.ell, sring.N
    assert host.shape == (L, 2, L, N)
    Ro = Ring(N, prime_size=[50] * L, primes=sring.primes, split_degree=1, engine=oracle_engine)
    sk = Polynomial(Ro).from_array(key.key[0])
    sk.to_NTT()
    q = np.array(sring.primes, dtype=object)[:, None]
    for i in range(L):
        a = poly_from_rows(Ro, host[i, 0])
        b = poly_from_rows(Ro, host[i, 1])
        a.repr = b.repr = sk.repr  # NTT domain
        phase = b - a * sk
        phase.to_coeff()
        msg = np.zeros((L, N), dtype=object)
        msg[i] = src_rows[i].astype(object) * (P % sring.primes[i]) % sring.primes[i]
        e = (phase.rows().astype(object) - msg) % q
        e = np.where(e > q // 2, e - q, e).astype(np.int64)
        assert (e == e[0]).all(), f"digit {i}: noise must be one integer per coefficient"
        assert np.abs(e[0]).max() <= 8 * 3.2


def test_gpu_keys_drive_batched_multiply_and_rotation(cuda):
    import torch

    from vfhe_b200.batch import CkksBatch, ciphertext_rows, gen_galois_key_batch, gen_rlk_batch, to_device, to_host
    from vfhe_b200.fhe import CKKS_Ciphertext
    from vfhe_b200.arith import repr
    from vfhe_b200.native import use_engine

    N = 2**12
    s, key, rng = _setup(cuda, N, 3, seed=22)
    step = 3
    with use_engine(cuda):
        z1 = [np.sqrt(rng.random(N // 2)) * np.exp(2j * np.pi * rng.random(N // 2)) for _ in range(2)]
        z2 = [np.sqrt(rng.random(N // 2)) * np.exp(2j * np.pi * rng.random(N // 2)) for _ in range(2)]
        c1 = [s.encrypt(s.encode(list(z)), key) for z in z1]
        c2 = [s.encrypt(s.encode(list(z)), key) for z in z2]
        for c in c1 + c2:
            c.to_NTT()
        rlk = gen_rlk_batch(s, key, lvl=0, engine=cuda)
        gk = gen_galois_key_batch(s, key, s.galois_gen(step), lvl=1, engine=cuda)
    special = s.special_rings[0].prime_indices[-1]
    t1 = to_device(np.stack([ciphertext_rows(c) for c in c1]))
    t2 = to_device(np.stack([ciphertext_rows(c) for c in c2]))
    prod = CkksBatch(s.rings[0], special).mul_relin_rescale(t1, t2, rlk)
    rot = CkksBatch(s.rings[1], special).rotate(prod, [s.galois_gen(step)] * 2, [gk, gk])
    torch.cuda.synchronize()
    hp, hr = to_host(prod), to_host(rot)
    delta = s.scaling_factor**2 / s.rings[0].primes[-1]
    with use_engine(cuda):
        for b in range(2):
            want = z1[b] * z2[b]
            for rows, expect in ((hp[b], want), (hr[b], np.roll(want, -step))):
                ct = CKKS_Ciphertext(s, lvl=1)
                ct.set_component_rows(0, rows[0])
                ct.set_component_rows(1, rows[1])
                ct.repr = repr.coeff
                dec = np.array(s.decode(s.decrypt(ct, key), scaling_factor=delta))
                assert np.abs(dec - expect).max() < 1e-4
