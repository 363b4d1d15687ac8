"""CKKS and CGGI16 over an engine.

Host-side mirror of the reference's ``vfhe.fhe`` surface
(modules/fhe/python/src/vfhe/fhe/ckks.py, cggi16.py).  Ciphertext arithmetic is
engine calls; CKKS encode/decode drive the engine's complex special FFT through
:mod:`vfhe_b200.complex` exactly as the reference does (on the cuda engine those
transforms run on the GPU with the reference's scalar rounding).
"""

from __future__ import annotations

import math

from .arith import Polynomial, Ring, ntt_processor, repr
from .complex import ComplexPolynomial, ComplexRing
from .mlwe import CMUX, LWE, MGSW_Scheme, MLWE, MLWE_Key, MLWE_Scheme, MLWE_Set
from .numbers import crt


class CKKS_Scheme(MLWE_Scheme):
    """CKKS (reference ckks.py:12-202)."""

    def __init__(self, rings, scaling_factor: float = 2**30, module_rank: int = 1, special_primes: int = 0,
                 special_rings=None):
        super().__init__(rings, special_primes=special_primes, special_rings=special_rings, module_rank=module_rank)
        self.scaling_factor = scaling_factor
        self.complex_ring = ComplexRing(self.ring.N // 2, True, engine=self.ring.engine)

    def encode(self, values) -> Polynomial:
        """Slots -> plaintext (ckks.py:37-56): IFFT, scale, round, NTT."""
        assert len(values) == self.ring.N // 2, f"Expected {self.ring.N // 2} values, got {len(values)}"
        c_poly = ComplexPolynomial(self.complex_ring)
        c_poly.from_array(values)
        c_poly.IFFT()
        c_poly *= self.scaling_factor
        poly = c_poly.round_to_RNS_cpp(self.ring)
        poly.rns_mask = self.ring.mask
        return poly

    def encode_batch(self, values_list) -> list[Polynomial]:
        """Many encodings in one engine call (complex_polys_ifft_scale_round_to_RNS_batch)."""
        polys = []
        for values in values_list:
            c = ComplexPolynomial(self.complex_ring)
            c.from_array(values)
            polys.append(c)
        out = self.complex_ring.exp_complex_polys_ifft_scale_round_to_RNS_batch(polys, self.ring,
                                                                                self.scaling_factor)
        for p in out:
            p.rns_mask = self.ring.mask
        return out

    def decode(self, poly: Polynomial, scaling_factor: float | None = None) -> list[complex]:
        """Plaintext -> slots (ckks.py:58-98): exact CRT, signed lift, FFT, 1/delta."""
        delta = self.scaling_factor if scaling_factor is None else scaling_factor
        mask = poly.rns_mask
        rns = poly.coeff_array()
        active = [(p, rns[i]) for i, (p, idx) in enumerate(zip(poly.ring.primes, poly.ring.prime_indices))
                  if (mask >> idx) & 1]
        primes = [p for p, _ in active]
        q = math.prod(primes)
        c_poly = ComplexPolynomial(self.complex_ring)
        half = poly.ring.N // 2
        coeffs = []
        for j in range(poly.ring.N):
            v = crt([int(r[j]) for _, r in active], primes)
            coeffs.append(float(v - q if v >= q // 2 else v))
        for i in range(half):
            c_poly[i] = complex(coeffs[i], coeffs[i + half])
        c_poly.FFT()
        return [v / delta for v in c_poly]

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
            return self.rational_rescale(ciphertext)
        dropped = math.prod(p for p in ciphertext.ring.primes if p not in nxt.primes)
        ciphertext.round_division(lvl=lvl + 1)
        ciphertext.delta = ciphertext.delta / dropped
        return ciphertext

    def rational_rescale(self, ct):
        """Rescale level lvl -> lvl + 1 when the next level is not a quotient of this one
        (reference ckks.py:150-202): each component is scaled and lifted into the union
        of both levels' primes (polynomial_RNSc_scaled_lift), then round-divided by the
        primes the next level drops; delta changes by prod(new) / prod(dropped)."""
        level = ct.lvl
        assert level < len(self.rings) - 1, "cannot rescale a ciphertext at the last level"
        start, end = ct.ring, self.rings[level + 1]
        pmap = ntt_processor(self.ring.engine).prime_to_index[(self.ring.N, self.ring.split_degree)]
        union = sorted(set(start.primes + end.primes), key=lambda p: pmap[p])
        union_ring = Ring(self.ring.N, primes=union, prime_size=[math.ceil(math.log2(p)) for p in union],
                          split_degree=self.ring.split_degree, engine=self.ring.engine)
        res = CKKS_Ciphertext(self, lvl=level + 1)
        for i in range(self.r):
            a = ct.get_a_poly(i).scaled_lift(union_ring).round_division(end)
            self.ring.lib.polynomial_copy_RNS_polynomial(res.obj_a_i(i), a.obj)
        b = ct.get_b_poly().scaled_lift(union_ring).round_division(end)
        self.ring.lib.polynomial_copy_RNS_polynomial(res.obj_b(), b.obj)
        self.ring.engine.check("rational_rescale")
        p_val = math.prod(p for p in end.primes if p not in start.primes)
        q_val = math.prod(q for q in start.primes if q not in end.primes)
        res.delta = ct.delta * p_val / q_val
        res.repr = repr.coeff
        return res


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
