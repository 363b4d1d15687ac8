"""Torus CGGI with FP64 FFT external products on the GPU against the exact-integer
oracle: the FFT product error, bit-exact key switching, blind rotations close to the
exact ones, and lookup-table decryptions identical to the table at full parameters
(n = 630, N = 1024, base 2^7 x 3, key switch base 2^2 x 8)."""

from __future__ import annotations

import numpy as np
import pytest

from tests.torus_helpers import oracle_bootstrap, oracle_external_product, oracle_keyswitch, torus_distance

pytestmark = pytest.mark.gpu


def _keys(n, N, seed):
    from vfhe_b200.cggi_fft import TorusKeys, TorusParams

    p = TorusParams(n=n, N=N)
    return p, TorusKeys.generate(p, np.random.default_rng(seed))


@pytest.mark.parametrize("N", [512, 1024, 2048])
def test_external_product_error(cuda, torus_oracle, N):
    import torch

    from vfhe_b200.cggi_fft import CggiFft, to_device, to_host

    p, keys = _keys(4, N, 10 + N)
    dev = CggiFft(keys, cuda)
    rng = np.random.default_rng(11)
    B = 6
    c = rng.integers(0, 1 << 32, (B, 2 * N), dtype=np.uint64).astype(np.uint32)
    out = torch.empty((B, 2 * N), dtype=torch.int32, device="cuda")
    frac = torch.empty(B, dtype=torch.float64, device="cuda")
    ffi = cuda.ffi
    ggsw_f = dev.bsk_f[: 2 * p.bs_levels * 2]  # GGSW(s_0) spectra
    dc = to_device(c)
    assert cuda.lib.vfhe_cuda_cggi_fft_external_product(
        ffi.cast("uint32_t*", out.data_ptr()), ffi.cast("uint32_t*", dc.data_ptr()), B,
        ffi.cast("double*", ggsw_f.data_ptr()), N, p.bs_base_log, p.bs_levels, ffi.cast("double*", frac.data_ptr()),
        ffi.cast("void*", torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    got = to_host(out)
    worst = 0
    for b in range(B):
        want = oracle_external_product(torus_oracle, c[b], keys.bsk[0], p)
        worst = max(worst, int(torus_distance(got[b], want).max()))
    # FP64 FFT of sums below 2^50: the rounded result is the exact product or next to it
    assert worst <= 1, worst
    assert float(frac.max()) < 0.5


def test_keyswitch_bit_exact(cuda, torus_oracle):
    from vfhe_b200.cggi_fft import CggiFft, to_device, to_host

    p, keys = _keys(630, 1024, 12)
    dev = CggiFft(keys, cuda)
    rng = np.random.default_rng(13)
    ext = rng.integers(0, 1 << 32, (40, p.N + 1), dtype=np.uint64).astype(np.uint32)
    got = to_host(dev.keyswitch(to_device(ext)))
    assert np.array_equal(got, oracle_keyswitch(torus_oracle, ext, keys.ksk, p))


def test_blind_rotation_close_to_exact(cuda, torus_oracle):
    from vfhe_b200.cggi_fft import CggiFft, test_vector, to_device, to_host

    p, keys = _keys(24, 1024, 14)
    dev = CggiFft(keys, cuda)
    rng = np.random.default_rng(15)
    lut = rng.integers(0, p.t, p.t)
    tv = test_vector(lut, p)
    m = rng.integers(0, p.t, 6)
    lwe = keys.encrypt(m, rng)
    got = to_host(dev.blind_rotate(to_device(lwe), to_device(tv)))
    want = oracle_bootstrap(torus_oracle, lwe, tv, keys.bsk, p)
    # each CMUX may round a coefficient to a neighbour of the exact value; the
    # difference stays far below the noise (2^-25 of the torus per key row)
    assert int(torus_distance(got, want).max()) < 1 << 12
    assert np.array_equal(keys.decrypt(got, keys.S), lut[m])
    assert np.array_equal(keys.decrypt(want, keys.S), lut[m])


def test_programmable_bootstrap_full_parameters(cuda):
    from vfhe_b200.cggi_fft import CggiFft, TorusKeys, TorusParams, test_vector, to_device, to_host

    p = TorusParams()
    rng = np.random.default_rng(16)
    keys = TorusKeys.generate(p, rng)
    dev = CggiFft(keys, cuda)
    lut = rng.integers(0, p.t, p.t)
    m = rng.integers(0, p.t, 2048)
    out = to_host(dev.bootstrap(to_device(keys.encrypt(m, rng)), to_device(test_vector(lut, p))))
    assert np.array_equal(keys.decrypt(out), lut[m])
    err = np.abs(keys.phases(out) - lut[m] * p.delta)
    assert err.max() < p.delta // 2  # every phase inside its box


def test_full_parameter_blind_rotation_matches_exact(cuda, torus_oracle):
    """n = 630: the GPU's FFT blind rotation and the exact-integer one decrypt alike and
    differ by far less than the bootstrapping noise."""
    from vfhe_b200.cggi_fft import CggiFft, test_vector, to_device, to_host

    p, keys = _keys(630, 1024, 17)
    dev = CggiFft(keys, cuda)
    rng = np.random.default_rng(18)
    lut = rng.integers(0, p.t, p.t)
    tv = test_vector(lut, p)
    m = rng.integers(0, p.t, 2)
    lwe = keys.encrypt(m, rng)
    got = to_host(dev.blind_rotate(to_device(lwe), to_device(tv)))
    want = oracle_bootstrap(torus_oracle, lwe, tv, keys.bsk, p)
    assert int(torus_distance(got, want).max()) < 1 << 14  # 2^-18 of the torus
    assert np.array_equal(keys.decrypt(got, keys.S), keys.decrypt(want, keys.S))
    assert np.array_equal(keys.decrypt(want, keys.S), lut[m])


def test_keyswitch_mismatches_come_from_key_noise(cuda, torus_oracle):
    """The rare lookup mismatches after the LWE key switch (about 4e-5 at these
    parameters) are a property of the key-switching key's noise, not of the GPU: for
    every mismatching sample the GPU's extracted LWE decrypts exactly as the
    exact-integer bootstrap's does (to the right table value), and the exact key switch
    of the GPU's extracted LWE equals the GPU's output bit for bit."""
    from vfhe_b200.cggi_fft import CggiFft, TorusKeys, TorusParams, test_vector, to_device, to_host

    p = TorusParams()
    rng = np.random.default_rng(41)
    keys = TorusKeys.generate(p, rng)
    dev = CggiFft(keys, cuda)
    lut = rng.integers(0, p.t, p.t)
    tv = test_vector(lut, p)
    tvd = to_device(tv)
    bad_idx, batches = [], 0
    while len(bad_idx) < 2 and batches < 8:
        m = rng.integers(0, p.t, 65536)
        lwe = keys.encrypt(m, rng)
        ext = dev.blind_rotate(to_device(lwe), tvd)
        out = to_host(dev.keyswitch(ext))
        ext = to_host(ext)
        assert (keys.decrypt(ext, keys.S) == lut[m]).all()  # the bootstrap itself never misses
        for i in np.nonzero(keys.decrypt(out) != lut[m])[0][:2]:
            bad_idx.append((lwe[i], ext[i], out[i], int(m[i])))
        batches += 1
    assert bad_idx, "no key-switch mismatch in 8 x 65536 samples"
    for lwe_i, ext_i, out_i, m_i in bad_idx:
        exact_ext = oracle_bootstrap(torus_oracle, lwe_i[None], tv, keys.bsk, p)
        assert keys.decrypt(exact_ext, keys.S)[0] == keys.decrypt(ext_i[None], keys.S)[0] == lut[m_i]
        assert np.array_equal(oracle_keyswitch(torus_oracle, ext_i[None], keys.ksk, p)[0], out_i)
