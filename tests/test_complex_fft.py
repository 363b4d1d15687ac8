"""CKKS special FFT (arith.cdef:84-93, complex.c): the engine's CT_NR / GS_RN /
bit_reverse_array / complex_poly_scale_double / round-to-RNS and the batched encoder
against the reference library, bit for bit (the reference's portable build rounds every
product and sum separately; so do the oracle and the GPU kernels)."""

from __future__ import annotations

import numpy as np
import pytest


def _raw(cp) -> np.ndarray:
    n2 = cp.ring.N2
    return np.frombuffer(cp.ring.ffi.buffer(cp.obj, 8 * n2), dtype=np.float64).copy()


def _transforms(engine, N, seed):
    from vfhe_b200.complex import ComplexPolynomial, ComplexRing

    ring = ComplexRing(N, engine=engine)
    rng = np.random.default_rng(seed)
    vals = rng.normal(size=N) + 1j * rng.normal(size=N)
    out = {}
    p = ComplexPolynomial(ring).from_array(vals)
    p.IFFT()
    out["ifft"] = _raw(p)
    p.FFT()
    out["fft_ifft"] = _raw(p)
    q = ComplexPolynomial(ring).from_array(vals)
    q *= 3.25
    out["scale"] = _raw(q)
    q.FFT()
    out["fft"] = _raw(q)
    return out


def _ckks(engine, N, seed):
    from vfhe_b200.arith import Ring, reset_registries
    from vfhe_b200.fhe import CKKS_Scheme
    from vfhe_b200.native import use_engine

    reset_registries()
    with use_engine(engine):
        R = Ring(N, prime_size=[50] + [40] * 3 + [50], split_degree=1)
        s = CKKS_Scheme(R, scaling_factor=2**40, special_primes=1)
        rng = np.random.default_rng(seed)
        zs = [np.sqrt(rng.random(N // 2)) * np.exp(2j * np.pi * rng.random(N // 2)) for _ in range(3)]
        enc = [s.encode(list(z)) for z in zs]
        rows = [e.rows() for e in enc]
        batch = [e.rows() for e in s.encode_batch([list(z) for z in zs])]
        dec = np.array(s.decode(enc[0]))
        return rows, batch, dec, zs[0]


def check_pair(engine, ref):
    for N in (8, 64, 1024):
        a, b = _transforms(engine, N, N), _transforms(ref, N, N)
        for k in a:
            assert np.array_equal(a[k].view(np.uint64), b[k].view(np.uint64)), (N, k)
    for N in (256, 2**12):
        rows, batch, dec, z = _ckks(engine, N, 7)
        rrows, rbatch, rdec, _ = _ckks(ref, N, 7)
        for x, y, bb in zip(rows, rrows, batch):
            assert np.array_equal(x, y)
            assert np.array_equal(bb, x)  # the batched encoder equals one-at-a-time encoding
        assert np.array_equal(dec.view(np.uint64), rdec.view(np.uint64))
        assert np.abs(dec - z).max() < 1e-6


def test_oracle_matches_reference(oracle_engine, ref_portable):
    check_pair(oracle_engine, ref_portable)


@pytest.mark.gpu
def test_cuda_matches_reference(cuda, ref_portable):
    check_pair(cuda, ref_portable)
