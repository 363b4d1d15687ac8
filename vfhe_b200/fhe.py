"""CKKS and CGGI16 over an engine.

Host-side mirror of the reference's ``vfhe.fhe`` surface
(modules/fhe/python/src/vfhe/fhe/ckks.py, cggi16.py).  Ciphertext arithmetic is
engine calls.  CKKS encode/decode are the client-side special FFT of
modules/arith/python/src/vfhe/arith/complex.py restated in numpy (the same roots,
stage order and scaling); they are approximate FP64 maps whose last bits may differ
from the reference's AVX-512 FMA kernels, which is why the parity tests inject the
encoded plaintext rather than re-encoding it on each engine.
"""

from __future__ import annotations

import functools
import math

import numpy as np

from .arith import Polynomial, Ring, repr
from .mlwe import CMUX, LWE, MGSW_Scheme, MLWE, MLWE_Key, MLWE_Scheme, MLWE_Set
from .numbers import crt


@functools.lru_cache(maxsize=16)
def special_roots(n2: int) -> tuple[np.ndarray, np.ndarray]:
    """CKKS "special" roots for the n2/4-slot FFT and their inverses (complex.py:90-106).

    Entry 2^(k-1)+i holds w^((5^brv(i)) n2 / 2^(k+1)) with w = exp(2 pi i / 2 n2);
    computed with 100-bit mpmath and rounded to complex128, as the reference does.
    """
    import mpmath as mp

    mp.mp.prec = 100
    w = mp.exp(2 * mp.pi * 1j / (2 * mp.mpf(n2)))
    res = [mp.mpc(1)] * n2
    logn = int(math.log2(n2))
    for k in range(logn - 1, 0, -1):
        for i in range(2 ** (k - 1)):
            b = int(bin(i)[2:].rjust(k - 1, "0")[::-1], 2) if k > 1 else 0
            e = ((5**b) * n2 // (2 ** (k + 1))) % (2 * n2)
            res[2 ** (k - 1) + i] = mp.power(w, e)
    fwd = np.array([complex(x) for x in res], dtype=np.complex128)
    inv = np.array([complex(x**-1) for x in res], dtype=np.complex128)
    return fwd, inv


def _brv_perm(n: int) -> np.ndarray:
    logn = int(math.log2(n))
    idx = np.arange(n)
    r = np.zeros(n, dtype=np.int64)
    for b in range(logn):
        r |= ((idx >> b) & 1) << (logn - 1 - b)
    return r


def _ct_nr(x: np.ndarray, ws: np.ndarray) -> None:
    n = x.size
    t, m = n, 1
    while m < n:
        t >>= 1
        for i in range(m):
            j1 = 2 * i * t
            v = x[j1 + t:j1 + 2 * t] * ws[m + i]
            x[j1 + t:j1 + 2 * t] = x[j1:j1 + t] - v
            x[j1:j1 + t] += v
        m <<= 1


def _gs_rn(x: np.ndarray, ws: np.ndarray) -> None:
    n = x.size
    t, m = 1, n
    while m > 1:
        h = m >> 1
        blk = x.reshape(h, 2 * t)
        u = blk[:, :t].copy()
        v = blk[:, t:].copy()
        blk[:, :t] = u + v
        blk[:, t:] = (u - v) * ws[h:2 * h, None]
        t <<= 1
        m >>= 1


def ckks_encode_coeffs(values, n_slots: int, delta: float) -> np.ndarray:
    """Slots -> rounded integer coefficients (ckks.py:37-56 with complex.py IFFT)."""
    z = np.zeros(n_slots, dtype=np.complex128)
    z[: len(values)] = np.asarray(values, dtype=np.complex128)
    _, inv = special_roots(2 * n_slots)
    z = z[np.argsort(_brv_perm(n_slots))]
    _gs_rn(z, inv)
    z = z * (1.0 / n_slots) * delta
    return np.concatenate([np.rint(z.real), np.rint(z.imag)]).astype(np.int64)


def ckks_decode_coeffs(coeffs: np.ndarray, delta: float) -> np.ndarray:
    """Signed coefficients -> slots (ckks.py:58-98 with complex.py FFT)."""
    n = coeffs.size // 2
    z = np.asarray(coeffs[:n], dtype=np.float64) + 1j * np.asarray(coeffs[n:], dtype=np.float64)
    fwd, _ = special_roots(2 * n)
    _ct_nr(z, fwd)
    z = z[_brv_perm(n)]
    return z / delta


class CKKS_Scheme(MLWE_Scheme):
    """CKKS (reference ckks.py:12-202)."""

    def __init__(self, rings, scaling_factor: float = 2**30, module_rank: int = 1, special_primes: int = 0,
                 special_rings=None):
        super().__init__(rings, special_primes=special_primes, special_rings=special_rings, module_rank=module_rank)
        self.scaling_factor = scaling_factor

    def encode(self, values) -> Polynomial:
        assert len(values) == self.ring.N // 2
        coeffs = ckks_encode_coeffs(values, self.ring.N // 2, self.scaling_factor)
        poly = Polynomial(self.ring).from_array(coeffs.tolist())
        poly.rns_mask = self.ring.mask
        return poly

    def decode(self, poly: Polynomial, scaling_factor: float | None = None) -> list[complex]:
        delta = self.scaling_factor if scaling_factor is None else scaling_factor
        mask = poly.rns_mask
        rns = poly.coeff_array()
        active = [(p, rns[i]) for i, (p, idx) in enumerate(zip(poly.ring.primes, poly.ring.prime_indices))
                  if (mask >> idx) & 1]
        primes = [p for p, _ in active]
        q = math.prod(primes)
        vals = np.empty(poly.ring.N, dtype=np.float64)
        for j in range(poly.ring.N):
            v = crt([int(r[j]) for _, r in active], primes)
            vals[j] = float(v - q if v >= q // 2 else v)
        return list(ckks_decode_coeffs(vals, delta))

    def encrypt(self, message: Polynomial, key: MLWE_Key, rng=None) -> CKKS_Ciphertext:
        out = CKKS_Ciphertext(self)
        self.sample(message, key, out=out, rng=rng)
        return out

    def decrypt(self, ciphertext: MLWE, key: MLWE_Key) -> Polynomial:
        return self.phase(ciphertext, key)

    def galois_gen(self, k: int) -> int:
        N = self.ring.N
        return pow(5, k % (N // 2), 2 * N)

    def rotate(self, ciphertext, k: int, ksk):
        return self.automorphism(ciphertext, self.galois_gen(k), ksk)

    def gen_rotation_key(self, key: MLWE_Key, k: int, rng=None):
        return self.gen_ksk_automorphism(key, key, self.galois_gen(k), rng=rng)

    def rescale(self, ciphertext):
        lvl = ciphertext.lvl
        assert lvl + 1 < len(self.rings), "no lower level to rescale into"
        nxt = self.rings[lvl + 1]
        if not nxt.is_quotient_ring(ciphertext.ring):
            raise NotImplementedError("non-nested level chains need rational rescaling")
        dropped = math.prod(p for p in ciphertext.ring.primes if p not in nxt.primes)
        ciphertext.round_division(lvl=lvl + 1)
        ciphertext.delta = ciphertext.delta / dropped
        return ciphertext


class CKKS_Ciphertext(MLWE):
    def __init__(self, scheme: CKKS_Scheme, lvl=None, ring=None, rank=None):
        super().__init__(scheme, lvl=lvl, ring=ring, rank=rank)
        self.delta = scheme.scaling_factor

    def _inherit(self, other) -> None:
        if isinstance(other, CKKS_Ciphertext):
            self.delta = other.delta

    def rescale(self):
        return self.scheme.rescale(self)

    def __mul__(self, other):
        if isinstance(other, CKKS_Ciphertext):
            assert self.scheme is other.scheme and self.ell == other.ell
            base = MLWE.__mul__(self, other)
            prod = CKKS_Ciphertext(self.scheme, lvl=base.lvl)
            prod.copy_from(base)
            prod.delta = self.delta * other.delta
            return self.scheme.rescale(prod)
        if isinstance(other, Polynomial):
            base = MLWE.__mul__(self, other)
            prod = CKKS_Ciphertext(self.scheme, lvl=base.lvl)
            prod.copy_from(base)
            prod.delta = self.delta * self.scheme.scaling_factor
            return self.scheme.rescale(prod)
        base = MLWE.__mul__(self, other)
        prod = CKKS_Ciphertext(self.scheme, lvl=base.lvl)
        prod.copy_from(base)
        prod.delta = self.delta
        return prod


CKKS_Scheme.ciphertext_type = CKKS_Ciphertext


class CGGI16_Key:
    def __init__(self) -> None:
        self.bk: list = []
        self.b_prec = 0


class CGGI16:
    """Functional bootstrap with RNS-gadget MGSW (reference cggi16.py:20-128)."""

    def __init__(self, scheme: MLWE_Scheme, gsw_ell: int | None = None):
        self.scheme = scheme
        self.mgsw_scheme = MGSW_Scheme(scheme, ell=gsw_ell)
        self.ring = scheme.ring

    def generate_bootstrap_key(self, input_key, output_key: MLWE_Key, rng=None) -> CGGI16_Key:
        bk = CGGI16_Key()
        lwe_key = input_key.extract_lwe_key() if isinstance(input_key, MLWE_Key) else input_key
        for s_i in lwe_key.get_s():
            poly = Polynomial(self.ring).from_array([s_i] + [0] * (self.ring.N - 1))
            m = self.mgsw_scheme.encrypt(poly, output_key, rng=rng)
            m.to_NTT()
            bk.bk.append(m)
        return bk

    @staticmethod
    def rotation_amounts(rlwe_in: LWE, N: int, torus_base: int) -> tuple[int, list[int]]:
        """(initial rotation, per-coefficient rotations) of the blind rotation (cggi16.py:49-79)."""
        q = math.prod(rlwe_in.ring.primes[: rlwe_in.l])
        b = crt(rlwe_in.get_b(), rlwe_in.ring.primes)
        a_rows = rlwe_in.get_a()
        a = [crt([a_rows[j][i] for j in range(rlwe_in.l)], rlwe_in.ring.primes) for i in range(rlwe_in.n)]
        offset = q // (4 * torus_base)
        rot_b = round(((b + offset) * (2 * N)) / q) % (2 * N)
        return (2 * N - rot_b) % (2 * N), [round((ai * (2 * N)) / q) % (2 * N) for ai in a]

    def functional_bootstrap_wo_extract(self, out: MLWE, tv: MLWE, rlwe_in: LWE, bk: CGGI16_Key, torus_base: int):
        N = self.ring.N
        rot_tv, rots = self.rotation_amounts(rlwe_in, N, torus_base)
        out.to_coeff()
        tv.to_coeff()
        lib = self.ring.lib
        lib.mlwe_RNSc_mul_by_xai(out.obj, tv.obj, rot_tv)
        self.ring.engine.check("mlwe_RNSc_mul_by_xai")
        out.repr = repr.coeff
        for i, a_i in enumerate(rots):
            if a_i == 0:
                continue
            out.to_coeff()
            rotated = MLWE(self.scheme)
            lib.mlwe_RNSc_mul_by_xai(rotated.obj, out.obj, a_i)
            rotated.repr = repr.coeff
            res = CMUX(out, rotated, bk.bk[i])
            out.copy_from(res)

    def LUT_packing(self, lut: list[int], size: int, LUT_prec: int) -> MLWE:
        tv = MLWE(self.scheme)
        N = self.ring.N
        q = self.ring.quotient_ring(ell=self.ring.ell).q_l
        scaled = [(v * q) // (1 << LUT_prec) for v in lut]
        coeffs = [scaled[i // (N // size)] if i // (N // size) < len(scaled) else 0 for i in range(N)]
        poly = Polynomial(self.scheme.rings[0]).from_bigint_array(coeffs)
        self.ring.lib.mlwe_RNS_trivial_sample_of_zero(tv.obj)
        tv.repr = repr.ntt
        tv += poly
        return tv

    def functional_bootstrap(self, out: LWE, tv: MLWE, rlwe_in: LWE, bk: CGGI16_Key, torus_base: int) -> None:
        rotated = MLWE(self.scheme)
        self.functional_bootstrap_wo_extract(rotated, tv, rlwe_in, bk, torus_base)
        rotated.to_coeff()
        obj = self.ring.lib.mlwe_extract_LWE(rotated.obj, 0)
        self.ring.engine.check("mlwe_extract_LWE")
        if out.obj is not None:
            self.ring.lib.free_lwe_sample(out.obj)
        out.obj = obj
        out.n = self.scheme.r * self.ring.N


__all__ = ["CKKS_Scheme", "CKKS_Ciphertext", "CGGI16", "CGGI16_Key", "MLWE_Set", "Ring"]
