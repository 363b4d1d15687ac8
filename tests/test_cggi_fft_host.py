"""Torus CGGI host logic and the exact oracle, without a GPU: key generation conventions,
encryption/decryption, exact negacyclic products and an exact programmable bootstrap
that decrypts to the lookup table."""

from __future__ import annotations

import numpy as np

from tests.torus_helpers import oracle_bootstrap, oracle_keyswitch, u32p

SMALL = dict(n=12, N=256, bs_base_log=7, bs_levels=3, ks_base_log=2, ks_levels=8, msg_bits=4)


def test_encrypt_decrypt_roundtrip():
    from vfhe_b200.cggi_fft import TorusKeys, TorusParams

    p = TorusParams(**SMALL)
    rng = np.random.default_rng(1)
    keys = TorusKeys.generate(p, rng)
    m = rng.integers(0, p.t, 200)
    assert np.array_equal(keys.decrypt(keys.encrypt(m, rng)), m)
    # noise is about sigma = 2^-15 of the torus
    ph = keys.phases(keys.encrypt(np.zeros(2000, dtype=np.int64), rng))
    assert 0.5 * 2**17 < ph.std() < 2 * 2**17


def test_negacyclic_times_binary_is_exact(torus_oracle):
    from vfhe_b200.cggi_fft import negacyclic_times_binary

    rng = np.random.default_rng(2)
    N = 128
    a = rng.integers(0, 1 << 32, (3, N), dtype=np.uint64).astype(np.uint32)
    S = rng.integers(0, 2, N).astype(np.int32)
    got = negacyclic_times_binary(a, S)
    for r in range(3):
        want = np.zeros(N, dtype=np.uint32)
        torus_oracle.tor_negacyclic_mac(u32p(want), S.ctypes.data_as(__import__("ctypes").POINTER(
            __import__("ctypes").c_int32)), u32p(np.ascontiguousarray(a[r])), N)
        assert np.array_equal(got[r], want)


def test_ggsw_rows_encrypt_the_gadget():
    from vfhe_b200.cggi_fft import TorusKeys, TorusParams, negacyclic_times_binary

    p = TorusParams(**SMALL)
    keys = TorusKeys.generate(p, np.random.default_rng(3))
    for i in range(3):
        for c in range(2):
            for lv in range(p.bs_levels):
                row = keys.bsk[i, c * p.bs_levels + lv]
                ph = (row[1].astype(np.int64) - negacyclic_times_binary(row[0], keys.S).astype(np.int64)) & 0xFFFFFFFF
                w = 1 << (32 - p.bs_base_log * (lv + 1))
                want = np.zeros(p.N, dtype=np.int64)
                # phase of row (c, l) = s_i w (-S for c = 0, 1 for c = 1), up to sigma 2^-25 noise
                if c == 1:
                    want[0] = keys.s[i] * w
                else:
                    want = -keys.s[i] * w * keys.S.astype(np.int64)
                err = (ph - want) & 0xFFFFFFFF
                err = np.minimum(err, (1 << 32) - err)
                assert err.max() < 2**12


def test_exact_bootstrap_decrypts_to_lut(torus_oracle):
    from vfhe_b200.cggi_fft import TorusKeys, TorusParams, test_vector

    p = TorusParams(**SMALL)
    rng = np.random.default_rng(4)
    keys = TorusKeys.generate(p, rng)
    lut = rng.integers(0, p.t, p.t)
    m = np.arange(p.t)
    lwe = keys.encrypt(m, rng)
    ext = oracle_bootstrap(torus_oracle, lwe, test_vector(lut, p), keys.bsk, p)
    assert np.array_equal(keys.decrypt(ext, keys.S), lut[m])
    ks = oracle_keyswitch(torus_oracle, ext, keys.ksk, p)
    assert np.array_equal(keys.decrypt(ks), lut[m])
