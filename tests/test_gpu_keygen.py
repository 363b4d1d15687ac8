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


def _cggi_setup(cuda, n, seed):
    from vfhe_b200.arith import Ring
    from vfhe_b200.fhe import CGGI16
    from vfhe_b200.mlwe import LWE_Key, MLWE_Scheme
    from vfhe_b200.native import use_engine

    with use_engine(cuda):
        rng = np.random.default_rng(seed)
        Rq = Ring(1024, prime_size=[50, 50, 50], split_degree=1)
        in_ring = Rq.quotient_ring(ell=2)
        s = MLWE_Scheme(Rq, special_primes=1, module_rank=1, max_lvl=1)
        key_s = [int(v) for v in rng.integers(0, 2, n)]
        out_key = s.key_gen_sparse(64, 3.2, ternary=False, rng=rng)
        cg = CGGI16(s)
        return s, cg, in_ring, key_s, LWE_Key(ring=in_ring, key=key_s, n=n), out_key, rng


def test_bootstrap_key_rows_decrypt_to_mgsw_messages(cuda, oracle_engine):
    """Every row of a GPU-made RNS CGGI16 bootstrapping key decrypts (on the CPU oracle)
    to its MGSW message plus one small integer shared by all limbs (mgsw.py:18-55)."""
    import torch

    from tests.helpers import poly_from_rows
    from vfhe_b200.arith import Polynomial, Ring
    from vfhe_b200.batch import gen_bootstrap_key_batch
    from vfhe_b200.native import use_engine

    n = 6
    s, cg, in_ring, key_s, in_key, out_key, rng = _cggi_setup(cuda, n, seed=31)
    with use_engine(cuda):
        bk = gen_bootstrap_key_batch(cg, in_key, out_key, engine=cuda)
    torch.cuda.synchronize()
    sring = cg.mgsw_scheme.ring
    L, N, ell = sring.ell, sring.N, cg.mgsw_scheme.ell
    host = bk.cpu().numpy().view(np.uint64)
    assert host.shape == (n, 2 * ell, 2, L, N)
    P = sring.modulus_ratio(s.rings[0])
    Ro = Ring(N, prime_size=[50] * L, primes=sring.primes, split_degree=1, engine=oracle_engine)
    so = Polynomial(Ro).from_array(out_key.key[0])
    so.to_NTT()
    q = np.array(sring.primes, dtype=object)[:, None]
    s_out = np.array(out_key.key[0], dtype=object)
    for k in range(n):
        for row in range(2 * ell):
            c, i = divmod(row, ell)
            a = poly_from_rows(Ro, host[k, row, 0])
            b = poly_from_rows(Ro, host[k, row, 1])
            a.repr = b.repr = so.repr
            phase = b - a * so
            phase.to_coeff()
            msg = np.zeros((L, N), dtype=object)
            f = P % sring.primes[i]
            if c == 0:  # -s_out s_k (P mod q_i) e_i
                msg[i] = (-s_out * key_s[k] * f) % sring.primes[i]
            else:       # s_k (P mod q_i) e_i: a constant
                msg[i, 0] = (key_s[k] * f) % sring.primes[i]
            e = (phase.rows().astype(object) - msg) % q
            e = np.where(e > q // 2, e - q, e).astype(np.int64)
            assert (e == e[0]).all(), (k, row)
            assert np.abs(e[0]).max() <= 8 * 3.2


def test_gpu_bootstrap_key_drives_batched_bootstrap(cuda):
    """LWEs bootstrapped with a GPU-made key decrypt to the lookup table."""
    import torch

    from vfhe_b200.batch import CggiBatch, gen_bootstrap_key_batch, to_device, to_host
    from vfhe_b200.mlwe import LWE, LWE_Key, encrypt_lwe
    from vfhe_b200.native import use_engine

    n, count, t = 64, 64, 16
    s, cg, in_ring, key_s, in_key, out_key, rng = _cggi_setup(cuda, n, seed=32)
    with use_engine(cuda):
        bk = gen_bootstrap_key_batch(cg, in_key, out_key, engine=cuda)
        lut = [int(v) for v in rng.integers(0, t, t)]
        tv = cg.LUT_packing(lut, t, 5)
        msgs = [int(v) for v in rng.integers(0, t, count)]
        lwes = [encrypt_lwe(in_ring, key_s, [round(m * in_ring.q_l / 32) % q for q in in_ring.primes], 3.2, rng)
                for m in msgs]
        tv.to_coeff()
        a = to_device(np.stack([np.array(x.get_a(), dtype=np.uint64) for x in lwes]))
        b = to_device(np.stack([np.array(x.get_b(), dtype=np.uint64) for x in lwes]))
        tvt = to_device(np.stack([tv.component_rows(0), tv.component_rows(1)]))
        oa, ob = CggiBatch(s, cuda).bootstrap(a, b, bk, tvt, t)
        torch.cuda.synchronize()
        ha, hb = to_host(oa), to_host(ob)
        ok = out_key.extract_lwe_key()
        key2 = LWE_Key(ring=in_ring, key=ok.get_s(), n=ok.n)
        for i in range(count):
            o = LWE(ring=in_ring, n=1024)
            o.set_rows(ha[i], hb[i])
            ph = o.phase(key2, recompose=True)
            assert round(ph * 32 / in_ring.q_l) % 32 == lut[msgs[i]]


def test_torus_device_keys_decrypt_and_bootstrap(cuda):
    """Torus keys drawn on the GPU: every bootstrapping-key row and key-switching-key
    row decrypts to its gadget message within 8 sigma, and 4096 programmable bootstraps
    with them decrypt to the lookup table."""
    import torch

    from vfhe_b200.cggi_fft import (CggiFft, TorusParams, generate_device_keys, lwe_dot, negacyclic_times_binary,
                                    test_vector, to_device, to_host)

    p = TorusParams()
    rng = np.random.default_rng(33)
    keys = generate_device_keys(p, rng, cuda)
    torch.cuda.synchronize()
    bsk = keys.bsk_d.cpu().numpy().view(np.uint32)
    ksk = keys.ksk_d.cpu().numpy().view(np.uint32)
    idx = rng.choice(p.n, 8, replace=False)
    for i in idx:
        for r in range(2 * p.bs_levels):
            c, lv = divmod(r, p.bs_levels)
            a = bsk[i, r, 0].astype(np.int64)
            b = bsk[i, r, 1].astype(np.int64)
            m = int(keys.s[i]) << (32 - p.bs_base_log * (lv + 1))
            a_plain = a.copy()
            if c == 0:  # the message sits in coefficient 0 of the mask
                a_plain[0] = (a_plain[0] - m) & 0xFFFFFFFF
            ph = (b - negacyclic_times_binary(a_plain.astype(np.uint32), keys.S).astype(np.int64)) & 0xFFFFFFFF
            ph[0] = (ph[0] - (m if c == 1 else 0)) & 0xFFFFFFFF
            e = np.where(ph >= 1 << 31, ph - (1 << 32), ph)
            assert np.abs(e).max() <= 8 * p.glwe_sigma * 2**32, (i, r)
    rows = ksk.reshape(-1, p.n + 1)
    ph = (rows[:, p.n].astype(np.int64) - lwe_dot(rows[:, :p.n], keys.s).astype(np.int64)) & 0xFFFFFFFF
    want = (keys.S[:, None].astype(np.int64) << (32 - p.ks_base_log * (np.arange(p.ks_levels)[None, :] + 1))).reshape(-1)
    e = (ph - want) & 0xFFFFFFFF
    e = np.where(e >= 1 << 31, e - (1 << 32), e)
    assert np.abs(e).max() <= 8 * p.lwe_sigma * 2**32
    assert abs(float(e.std()) / (p.lwe_sigma * 2**32) - 1.0) < 0.1
    dev = CggiFft(keys, cuda)
    lut = rng.integers(0, p.t, p.t)
    tv = to_device(test_vector(lut, p))
    msgs = rng.integers(0, p.t, 4096)
    ext = dev.blind_rotate(to_device(keys.encrypt(msgs, rng)), tv)
    torch.cuda.synchronize()
    assert (keys.decrypt(to_host(ext), keys.S) == lut[msgs]).all()


def test_key_files_save_load_use(cuda, tmp_path):
    """Keys saved to key files and loaded back are identical and drive the same results."""
    import torch

    from vfhe_b200 import keyfile
    from vfhe_b200.batch import CkksBatch, ciphertext_rows, gen_rlk_batch, to_device
    from vfhe_b200.cggi_fft import CggiFft, TorusParams, generate_device_keys, test_vector
    from vfhe_b200.cggi_fft import to_device as to_device32
    from vfhe_b200.native import use_engine

    s, key, rng = _setup(cuda, 2**12, 3, seed=34)
    N = 2**12
    with use_engine(cuda):
        rlk = gen_rlk_batch(s, key, lvl=0, engine=cuda)
        cts = [s.encrypt(s.encode(list(np.exp(2j * np.pi * rng.random(N // 2)))), key) for _ in range(4)]
        for c in cts:
            c.to_NTT()
    sring = s.special_rings[0]
    keyfile.save(tmp_path / "rlk.vfhekey", rlk, keyfile.KSK, moduli=sring.primes, aux=(0, 0, N, 1))
    h, rlk2 = keyfile.load(tmp_path / "rlk.vfhekey", engine=cuda)
    assert h.kind == keyfile.KSK and h.moduli == list(sring.primes) and torch.equal(rlk, rlk2)
    special = sring.prime_indices[-1]
    t1 = to_device(np.stack([ciphertext_rows(c) for c in cts[0::2]]))
    t2 = to_device(np.stack([ciphertext_rows(c) for c in cts[1::2]]))
    batch = CkksBatch(s.rings[0], special)
    assert torch.equal(batch.mul_relin_rescale(t1, t2, rlk), batch.mul_relin_rescale(t1, t2, rlk2))

    p = TorusParams()
    keys = generate_device_keys(p, np.random.default_rng(35), cuda)
    keyfile.save(tmp_path / "tbsk.vfhekey", keys.bsk_d, keyfile.TORUS_BSK, aux=(p.bs_base_log, p.bs_levels))
    keyfile.save(tmp_path / "tksk.vfhekey", keys.ksk_d, keyfile.TORUS_KSK, aux=(p.ks_base_log, p.ks_levels))
    _, b2 = keyfile.load(tmp_path / "tbsk.vfhekey", engine=cuda)
    _, k2 = keyfile.load(tmp_path / "tksk.vfhekey", engine=cuda)
    assert torch.equal(b2, keys.bsk_d) and torch.equal(k2, keys.ksk_d)
    dev1 = CggiFft(keys, cuda)
    keys.bsk_d, keys.ksk_d = b2, k2
    dev2 = CggiFft(keys, cuda)
    lut = rng.integers(0, p.t, p.t)
    tv = to_device32(test_vector(lut, p))
    lwe = to_device32(keys.encrypt(rng.integers(0, p.t, 256), rng))
    assert torch.equal(dev1.bootstrap(lwe, tv), dev2.bootstrap(lwe, tv))
