"""(M)LWE schemes, keys, key-switching key sets, MGSW and LWE over an engine.

Host-side mirror of the reference's ``vfhe.mlwe`` surface
(modules/mlwe/python/src/vfhe/mlwe/mlwe.py, mgsw.py, lwe.py): same classes, method
names and level conventions; each operation is one call into the engine.

Sampling: without ``rng`` a sample draws from the engine's own random stream, as in
the reference.  With a numpy ``Generator`` the uniform ``a`` and the rounded-Gaussian
error are drawn on the host and the sample is assembled with deterministic engine
operations (NTT, ring products, additions), so every engine given the same seed
produces bit-identical keys and ciphertexts.  The parity tests and the benchmark use
that path.
"""

from __future__ import annotations

import contextlib
import secrets
from collections.abc import Sequence

import numpy as np

from .arith import Polynomial, Ring, repr
from .numbers import crt


class PolyView(Polynomial):
    """Non-owning view of a polynomial held inside an engine struct."""

    def __init__(self, ring: Ring, handle, rep=repr.empty) -> None:  # noqa: D107
        self.ring = ring
        self.obj = handle
        self.repr = rep

    def __del__(self) -> None:
        pass


def _mask_of(ring: Ring) -> int:
    return ring.mask


class MLWE_Scheme:
    """Leveled scheme (reference mlwe.py:31-89)."""

    ciphertext_type: type

    def __init__(
        self,
        rings: list[Ring] | Ring,
        special_primes: int = 0,
        special_rings: list[Ring] | None = None,
        max_lvl: int | None = None,
        module_rank: int = 1,
    ) -> None:
        if isinstance(rings, Ring):
            max_lvl = max_lvl if max_lvl is not None else len(rings.primes) - 1
            if special_primes == 0:
                self.rings = [rings.quotient_ring(ell=rings.ell - i) for i in range(max_lvl)]
                self.special_rings = self.rings
            else:
                self.rings = [rings.quotient_ring(ell=rings.ell - i) for i in range(special_primes, special_primes + max_lvl)]
                special_mask = ((1 << special_primes) - 1) << self.rings[0].ell
                self.special_rings = [rings.quotient_ring(mask=self.rings[i].mask | special_mask) for i in range(len(self.rings))]
        else:
            max_lvl = max_lvl if max_lvl is not None else len(rings)
            special_rings = special_rings if special_rings is not None else rings
            self.rings = [rings[i] for i in range(max_lvl)]
            self.special_rings = [special_rings[i] for i in range(max_lvl)]
        self.r = module_rank
        self.N = self.rings[0].N
        self.ell = len(self.rings)
        self.max_lvl = max_lvl
        self.rlk = None

    @property
    def ring(self) -> Ring:
        return self.rings[0]

    @property
    def engine(self):
        return self.rings[0].engine

    @property
    def extended_rank(self) -> int:
        return self.r * (self.r + 3) // 2

    @property
    def special_primes(self) -> int:
        return self.special_rings[0].ell - self.rings[0].ell if self.special_rings and self.rings else 0

    def level_of_ring(self, ring: Ring, strict: bool = True) -> int:
        for lvl, r in enumerate(self.rings):
            if r.mask == ring.mask:
                return lvl
        if strict:
            raise ValueError("ring is not one of the scheme's levels; pass lvl explicitly")
        return -1

    # -- keys
    def key_gen_sparse(self, h: int, sigma_err: float, ternary: bool = True, rng: np.random.Generator | None = None):
        """Sparse key with h nonzero coefficients (reference mlwe.py:130-143)."""
        assert self.N * self.r >= h
        key = [[0] * self.N for _ in range(self.r)]
        placed, sign = 0, 1
        while placed < h:
            pos = int(rng.integers(0, self.N * self.r)) if rng is not None else secrets.randbelow(self.N * self.r)
            if key[pos // self.N][pos % self.N]:
                continue
            key[pos // self.N][pos % self.N] = sign
            if ternary:
                sign = -sign
            placed += 1
        return MLWE_Key(key, sigma_err, self)

    def key_gen_uniform_ternary(self, sigma_err: float, rng: np.random.Generator):
        key = [[int(v) for v in rng.integers(-1, 2, self.N)] for _ in range(self.r)]
        return MLWE_Key(key, sigma_err, self)

    def _gen_ksk_components(self, key_out: MLWE_Key, key_poly: list[Polynomial], lvl: int, rng=None):
        """Gadget ciphertexts of key_poly[j] * (P mod q_i) e_i (reference mlwe.py:145-177)."""
        sring = self.special_rings[lvl]
        special_q = sring.modulus_ratio(self.rings[lvl])
        key_out_special = MLWE_Key(key_out.key, key_out.sigma_err, self, ring=sring)
        result = []
        for poly_j in key_poly:
            if poly_j.ring != sring:
                poly_j = Polynomial(sring).from_bigint_array(poly_j.get_polynomial(signed=True))
            comps = []
            for i in range(sring.ell):
                factor = [0] * i + [special_q % sring.primes[i]] + [0] * (sring.ell - 1 - i)
                out = MLWE(self, lvl=lvl, ring=sring)
                self.sample(poly_j * factor, key_out_special, out=out, rng=rng)
                comps.append(out)
            result.append(comps)
        return result

    def gen_ksk_for_level(self, key_out, key_in, lvl: int, rng=None):
        polys = key_in if isinstance(key_in, list) else key_in.poly
        return MLWE_Set(self._gen_ksk_components(key_out, polys, lvl, rng))

    def gen_rlk_for_level(self, key_out, quad_polys, lvl: int, rng=None):
        return MLWE_Set(self._gen_ksk_components(key_out, quad_polys, lvl, rng) + [None] * self.r)

    def quadratic_key_polys(self, key: MLWE_Key) -> list[Polynomial]:
        return [-(key.poly[i] * key.poly[j]) for i in range(self.r) for j in range(i, self.r)]

    def gen_rlk(self, key_out, quad_polys, lvl: int | None = None, rng=None):
        quad = quad_polys if isinstance(quad_polys, list) else self.quadratic_key_polys(quad_polys)
        assert len(quad) == self.r * (self.r + 1) // 2
        if lvl is not None:
            return self.gen_rlk_for_level(key_out, quad, lvl, rng)
        return [self.gen_rlk_for_level(key_out, quad, l, rng) for l in range(len(self.rings))]

    def gen_ksk(self, key_out, key_in, lvl: int | None = None, rng=None):
        polys = key_in if isinstance(key_in, list) else key_in.poly
        if lvl is not None:
            return self.gen_ksk_for_level(key_out, polys, lvl, rng)
        return [self.gen_ksk_for_level(key_out, polys, l, rng) for l in range(len(self.rings))]

    def gen_ksk_automorphism(self, key_out, key_in, g: int, lvl: int | None = None, rng=None):
        perm = [p.automorphism(g) for p in key_in.poly]
        return self.gen_ksk(key_out, perm, lvl, rng)

    # -- evaluation
    def keyswitch(self, c, ksk):
        ksk = ksk if isinstance(ksk, MLWE_Set) else ksk[c.lvl]
        out = c.new_like(lvl=c.lvl, ring=self.special_rings[c.lvl])
        c.to_coeff()
        self.engine.lib.mlwe_RNSc_GHS_hybrid_keyswitch(out.obj, c.obj, ksk.obj, c.lvl)
        self.engine.check("mlwe_RNSc_GHS_hybrid_keyswitch")
        out.repr = repr.coeff
        out.ring = self.rings[c.lvl]
        return out

    def automorphism(self, c, gen: int, ksk):
        ksk = ksk if isinstance(ksk, MLWE_Set) else ksk[c.lvl]
        out = c.new_like(lvl=c.lvl, ring=self.special_rings[c.lvl])
        c.to_coeff()
        self.engine.lib.mlwe_automorphism_RNSc_GHS(out.obj, c.obj, gen, ksk.obj, c.lvl)
        self.engine.check("mlwe_automorphism_RNSc_GHS")
        out.repr = repr.coeff
        out.ring = self.rings[c.lvl]
        return out

    def sample(self, msg: Polynomial, key: MLWE_Key, out=None, lvl: int | None = None, rng=None):
        """Encrypt msg under key (reference mlwe.py:343-366; mlwe.c:190-241)."""
        if not out:
            out = self.ciphertext_type(self, lvl=lvl)
        msg.to_coeff()
        lib = self.engine.lib
        if rng is None:
            lib.mlwe_RNSc_sample(out.obj, key.obj, msg.obj)
            self.engine.check("mlwe_RNSc_sample")
        else:
            ring = out.ring
            e = np.rint(rng.normal(0.0, key.sigma_err, ring.N)).astype(np.int64)
            b = out.component(out.r)
            lib.int_array_to_RNS(b.obj, self.engine.ffi.from_buffer("uint64_t[]", e.view(np.uint64)))
            tmp = Polynomial(ring)
            for i in range(out.r):
                a = out.component(i)
                a.set_rows(np.stack([rng.integers(0, q, ring.N, dtype=np.uint64) for q in ring.primes]))
                a.rns_mask = ring.mask
                lib.polynomial_RNSc_to_RNS(a.obj, a.obj)
                lib.polynomial_mul_RNS_polynomial(tmp.obj, key.s_handle(i), a.obj)
                lib.polynomial_add_RNS_polynomial(b.obj, b.obj, tmp.obj)
            lib.mlwe_RNS_to_RNSc(out.obj, out.obj)
            lib.polynomial_add_RNSc_polynomial(b.obj, b.obj, msg.obj)
            self.engine.check("sample")
        out.repr = repr.coeff
        return out

    def phase(self, c, key: MLWE_Key, out: Polynomial | None = None) -> Polynomial:
        out = out or Polynomial(c.ring)
        k = key if key.ring == c.ring else MLWE_Key(key.key, key.sigma_err, self, ring=c.ring)
        c.to_NTT()
        self.engine.lib.mlwe_RNS_phase(out.obj, c.obj, k.obj)
        self.engine.check("mlwe_RNS_phase")
        out.repr = repr.ntt
        return out

    def tensor_product(self, in1, in2) -> list[Polynomial]:
        assert in1.ring == in2.ring
        in1.to_NTT()
        in2.to_NTT()
        outs = [Polynomial(in1.ring, repr.ntt) for _ in range(self.extended_rank + 1)]
        ptrs = self.engine.ffi.new("void*[]", [p.obj for p in outs])
        self.engine.lib.mlwe_tensor_product(ptrs, in1.obj, in2.obj)
        self.engine.check("mlwe_tensor_product")
        return outs

    def multiply(self, in1, in2, ksk=None):
        """Tensor and (with ksk) relinearise (reference mlwe.py:415-455; mlwe.c:711-760)."""
        assert in1.ring == in2.ring and in1.lvl == in2.lvl
        in1.to_NTT()
        in2.to_NTT()
        lib = self.engine.lib
        if ksk is None:
            out = in1.new_like(lvl=in1.lvl, rank=self.extended_rank)
            out.is_extended = True
            lib.mlwe_multiply(out.obj, in1.obj, in2.obj, self.engine.ffi.NULL)
            self.engine.check("mlwe_multiply")
            out.repr = repr.ntt
            return out
        ksk = ksk if isinstance(ksk, MLWE_Set) else ksk[in1.lvl]
        out = in1.new_like(lvl=in1.lvl, ring=self.special_rings[in1.lvl])
        lib.mlwe_multiply(out.obj, in1.obj, in2.obj, ksk.obj)
        self.engine.check("mlwe_multiply")
        out.repr = repr.ntt
        out.ring = self.rings[in1.lvl]
        return out

    def relinearize(self, c_ext, ksk):
        ksk = ksk if isinstance(ksk, MLWE_Set) else ksk[c_ext.lvl]
        out = c_ext.new_like(lvl=c_ext.lvl, ring=self.special_rings[c_ext.lvl])
        c_ext.to_coeff()
        self.engine.lib.mlwe_RNSc_GHS_hybrid_keyswitch(out.obj, c_ext.obj, ksk.obj, c_ext.lvl)
        self.engine.check("relinearize")
        out.repr = repr.coeff
        out.ring = self.rings[c_ext.lvl]
        return out


class MLWE_Key:
    """Secret key at a ring (reference mlwe.py:474-518)."""

    def __init__(self, key: list[list[int]], sigma_err: float, scheme: MLWE_Scheme, ring: Ring | None = None):
        assert len(key) == scheme.r
        self.key = key
        self.scheme = scheme
        self.sigma_err = sigma_err
        self.ring = ring if ring is not None else scheme.rings[0]
        eng = self.ring.engine
        flat = np.array([int(x) & 0xFFFFFFFFFFFFFFFF for row in key for x in row], dtype=np.uint64)
        self.obj = eng.lib.mlwe_new_RNS_key_from_array(
            eng.ffi.from_buffer("uint64_t[]", flat), self.ring.N, scheme.r, self.ring.ell, self.ring.NTT, sigma_err
        )
        eng.check("mlwe_new_RNS_key_from_array")
        self.poly = [Polynomial(self.ring).from_array(s) for s in key]
        st = eng.ffi.cast("RNS_MLWE_Key", self.obj)
        for i in range(scheme.r):
            eng.lib.polynomial_copy_RNS_polynomial(st.s_RNS[i], self.poly[i].obj)
        eng.check("MLWE_Key")

    def s_handle(self, i: int):
        return self.ring.ffi.cast("RNS_MLWE_Key", self.obj).s_RNS[i]

    def __del__(self) -> None:
        with contextlib.suppress(Exception):
            self.ring.lib.free_mlwe_RNS_key(self.obj)

    def extract_lwe_key(self) -> LWE_Key:
        flat = [x for row in self.key for x in row]
        return LWE_Key(ring=self.scheme.rings[0], key=flat, n=len(flat))


class MLWE_Set:
    """Key-switching key set passed to C as ``void*[]`` (reference mlwe.py:521-555)."""

    def __init__(self, mlwe: Sequence[list | None] | None = None):
        if mlwe is None:
            return
        self.mlwe = mlwe
        self.dim = 2
        eng = next(c for c in mlwe if c is not None)[0].ring.engine
        self.engine = eng
        self.obj = eng.ffi.new("void*[]", len(mlwe))
        self._keep = []
        for j, comp in enumerate(mlwe):
            if comp is None:
                self.obj[j] = eng.ffi.NULL
                continue
            for x in comp:
                x.to_NTT()
            tmp = eng.ffi.new("void*[]", [c.obj for c in comp])
            self.obj[j] = eng.lib.mlwe_create_copy_array(tmp, len(comp))
            eng.check("mlwe_create_copy_array")

    @staticmethod
    def flatten_array(array: list[MLWE_Set]) -> MLWE_Set:
        out = MLWE_Set()
        out.mlwe = [a.mlwe for a in array]
        out.dim = array[0].dim + 1
        eng = array[0].engine
        out.engine = eng
        out.obj = eng.ffi.new("void*[]", len(array))
        out._children = array
        for j, a in enumerate(array):
            out.obj[j] = eng.ffi.cast("void *", a.obj)
        return out

    def key_arrays(self) -> list[np.ndarray | None]:
        """Digit-major NTT-domain key material [digits][2][limbs][N] per component."""
        res = []
        for comp in self.mlwe:
            if comp is None:
                res.append(None)
                continue
            res.append(np.stack([np.stack([c.component(i).rows() for i in range(c.r + 1)]) for c in comp]))
        return res


class MLWE:
    """MLWE ciphertext (reference mlwe.py:558-841)."""

    def __init__(self, scheme: MLWE_Scheme, lvl: int | None = None, ring: Ring | None = None, rank: int | None = None):
        if lvl is None:
            lvl = scheme.level_of_ring(ring, strict=False) if ring is not None else 0
        if ring is None:
            ring = scheme.rings[lvl]
        self.r = rank if rank is not None else scheme.r
        self.obj = ring.lib.mlwe_alloc_RNS_sample(ring.N, self.r, ring.mask, ring.NTT)
        ring.engine.check("mlwe_alloc_RNS_sample")
        self.ring = ring
        self.scheme = scheme
        self.repr = repr.empty
        self.lvl = lvl
        self.is_extended = False

    @property
    def ell(self) -> int:
        return self.ring.ell

    @property
    def _eng(self):
        return self.ring.engine

    def new_like(self, lvl=None, ring=None, rank=None):
        out = type(self)(self.scheme, lvl=self.lvl if lvl is None else lvl, ring=ring, rank=rank)
        out._inherit(self)
        return out

    def _inherit(self, other) -> None:
        pass

    def __del__(self) -> None:
        with contextlib.suppress(Exception):
            self.ring.lib.free_mlwe_RNS_sample(self.obj)

    # -- component access
    def component(self, i: int) -> PolyView:
        """a_i for i < r, b for i == r, as a non-owning polynomial view."""
        st = self.ring.ffi.cast("RNS_MLWE", self.obj)
        h = st.b if i == self.r else st.a[i]
        return PolyView(self.ring, h, self.repr)

    def set_component_rows(self, i: int, rows: np.ndarray) -> None:
        v = self.component(i)
        v.set_rows(rows)
        v.rns_mask = self.ring.mask

    def component_rows(self, i: int) -> np.ndarray:
        return self.component(i).rows()

    def obj_a_i(self, j: int):
        return self.ring.ffi.cast("RNS_MLWE", self.obj).a[j]

    def obj_b(self):
        return self.ring.ffi.cast("RNS_MLWE", self.obj).b

    # -- representation
    def to_NTT(self) -> None:
        if self.repr == repr.ntt:
            return
        self.ring.lib.mlwe_RNSc_to_RNS(self.obj, self.obj)
        self._eng.check("mlwe_RNSc_to_RNS")
        self.repr = repr.ntt

    def to_coeff(self) -> None:
        if self.repr == repr.coeff:
            return
        self.ring.lib.mlwe_RNS_to_RNSc(self.obj, self.obj)
        self._eng.check("mlwe_RNS_to_RNSc")
        self.repr = repr.coeff

    # -- arithmetic
    def multiply_poly(self, in_rlwe, in_poly) -> None:
        assert in_rlwe.repr == in_poly.repr == repr.ntt
        self.ring.lib.mlwe_RNS_mul_by_poly(self.obj, in_rlwe.obj, in_poly.obj)
        self._eng.check("mlwe_RNS_mul_by_poly")
        self.repr = repr.ntt

    def multiply_scalar(self, in_rlwe, pointer_to_int_list) -> None:
        if self is not in_rlwe:
            self.ring.lib.mlwe_copy_RNS_sample(self.obj, in_rlwe.obj)
        self.ring.lib.mlwe_scale_RNS_mlwe_RNS(self.obj, pointer_to_int_list)
        self._eng.check("mlwe_scale_RNS_mlwe_RNS")
        self.repr = in_rlwe.repr

    def add_MLWE(self, in1, in2) -> None:
        assert in1.repr == in2.repr
        self.ring.lib.mlwe_add_RNSc_sample(self.obj, in1.obj, in2.obj)
        self._eng.check("mlwe_add_RNSc_sample")
        self.repr = in1.repr

    def sub_MLWE(self, in1, in2) -> None:
        assert in1.repr == in2.repr
        self.ring.lib.mlwe_sub_RNSc_sample(self.obj, in1.obj, in2.obj)
        self._eng.check("mlwe_sub_RNSc_sample")
        self.repr = in1.repr

    def add_poly(self, in1, in2) -> None:
        assert in1.repr == in2.repr
        f = self.ring.lib.mlwe_RNS_add_polynomial if in1.repr == repr.ntt else self.ring.lib.mlwe_add_RNSc_polynomial
        f(self.obj, in1.obj, in2.obj)
        self._eng.check("mlwe_add_polynomial")
        self.repr = in1.repr

    def sub_poly(self, in1, in2) -> None:
        assert in1.repr == in2.repr
        f = self.ring.lib.mlwe_RNS_sub_polynomial if in1.repr == repr.ntt else self.ring.lib.mlwe_sub_RNSc_polynomial
        f(self.obj, in1.obj, in2.obj)
        self._eng.check("mlwe_sub_polynomial")
        self.repr = in1.repr

    def mul_by_xai(self, a: int, minus1: bool = False):
        """self * X^a (or self * (X^a - 1)), coefficient domain."""
        self.to_coeff()
        out = self.new_like()
        f = self.ring.lib.mlwe_RNSc_mul_by_xai_minus1 if minus1 else self.ring.lib.mlwe_RNSc_mul_by_xai
        f(out.obj, self.obj, a)
        self._eng.check("mlwe_RNSc_mul_by_xai")
        out.repr = repr.coeff
        return out

    def get_a_poly(self, j: int) -> Polynomial:
        res = Polynomial(self.ring)
        self.ring.lib.polynomial_copy_RNS_polynomial(res.obj, self.obj_a_i(j))
        res.repr = self.repr
        return res

    def get_b_poly(self) -> Polynomial:
        res = Polynomial(self.ring)
        self.ring.lib.polynomial_copy_RNS_polynomial(res.obj, self.obj_b())
        res.repr = self.repr
        return res

    def copy(self):
        res = self.new_like()
        self.ring.lib.mlwe_copy_RNS_sample(res.obj, self.obj)
        self._eng.check("mlwe_copy_RNS_sample")
        res.repr = self.repr
        return res

    __copy__ = copy

    def copy_from(self, other) -> None:
        self.ring.lib.mlwe_copy_RNS_sample(self.obj, other.obj)
        self._eng.check("mlwe_copy_RNS_sample")
        self.repr = other.repr

    def round_division(self, ring: Ring | None = None, lvl: int | None = None):
        assert (ring is None) != (lvl is None)
        if lvl is None:
            lvl = self.scheme.level_of_ring(ring)
        else:
            ring = self.scheme.rings[lvl]
        assert ring.is_quotient_ring(self.ring)
        self.to_coeff()
        self.ring.lib.mlwe_round_division_RNSc(self.obj, self.ring.mask ^ ring.mask)
        self._eng.check("mlwe_round_division_RNSc")
        self.lvl = lvl
        self.ring = ring
        return self

    def __add__(self, other):
        if isinstance(other, int):
            if other == 0:
                return self.copy()
            raise NotImplementedError
        if self.repr != other.repr:
            self.to_NTT()
            other.to_NTT()
        res = self.new_like()
        if isinstance(other, MLWE):
            res.add_MLWE(self, other)
        else:
            res.add_poly(self, other)
        return res

    __radd__ = __add__

    def __iadd__(self, other):
        if isinstance(other, int):
            if other == 0:
                return self
            raise NotImplementedError
        if self.repr != other.repr:
            self.to_NTT()
            other.to_NTT()
        if isinstance(other, MLWE):
            self.add_MLWE(self, other)
        else:
            self.add_poly(self, other)
        return self

    def __sub__(self, other):
        if isinstance(other, int):
            if other == 0:
                return self.copy()
            raise NotImplementedError
        if self.repr != other.repr:
            self.to_NTT()
            other.to_NTT()
        res = self.new_like()
        if isinstance(other, MLWE):
            res.sub_MLWE(self, other)
        else:
            res.sub_poly(self, other)
        return res

    def __isub__(self, other):
        if self.repr != other.repr:
            self.to_NTT()
            other.to_NTT()
        if isinstance(other, MLWE):
            self.sub_MLWE(self, other)
        else:
            self.sub_poly(self, other)
        return self

    def __mul__(self, other):
        if isinstance(other, Polynomial):
            res = self.new_like()
            o = other if other.ring == self.ring else other.base_extend(self.ring)
            self.to_NTT()
            o.to_NTT()
            res.multiply_poly(self, o)
            return res
        if isinstance(other, MGSW):
            return other * self
        if isinstance(other, MLWE):
            assert self.scheme.rlk is not None, "Relinearization key (rlk) must be set in the scheme"
            return self.scheme.multiply(self, other, self.scheme.rlk)
        res = self.new_like()
        res.multiply_scalar(self, other)
        return res

    __rmul__ = __mul__


MLWE_Scheme.ciphertext_type = MLWE


class MGSW_Scheme:
    """RNS MGSW over an MLWE scheme (reference mgsw.py:12-55)."""

    def __init__(self, mlwe_scheme: MLWE_Scheme, ell: int | None = None):
        self.mlwe_scheme = mlwe_scheme
        self.ell = ell if ell else mlwe_scheme.rings[0].ell
        self.ring = mlwe_scheme.special_rings[0]

    def encrypt(self, msg: Polynomial, key: MLWE_Key, lvl: int = 0, rng=None) -> MGSW:
        special_q = self.ring.modulus_ratio(self.mlwe_scheme.rings[lvl])
        if msg.ring != self.ring:
            msg = msg.base_extend(self.ring)
        key_special = MLWE_Key(key.key, key.sigma_err, self.mlwe_scheme, ring=self.ring)
        result = []
        for j in range(self.mlwe_scheme.r):
            sm = -key.poly[j] * msg
            if sm.ring != self.ring:
                sm = sm.base_extend(self.ring)
            for i in range(self.ell - lvl):
                factor = [0] * i + [special_q % self.ring.primes[i]] + [0] * (self.ring.ell - 1 - i)
                out = MLWE(self.mlwe_scheme, ring=self.ring)
                self.mlwe_scheme.sample(sm * factor, key_special, out=out, rng=rng)
                result.append(out)
        for i in range(self.ell - lvl):
            factor = [0] * i + [special_q % self.ring.primes[i]] + [0] * (self.ring.ell - 1 - i)
            out = MLWE(self.mlwe_scheme, ring=self.ring)
            self.mlwe_scheme.sample(msg * factor, key_special, out=out, rng=rng)
            result.append(out)
        return MGSW(self, obj=result)


class MGSW:
    def __init__(self, scheme: MGSW_Scheme, obj: list[MLWE] | None = None):
        self.scheme = scheme
        self.obj = obj if obj else [
            MLWE(scheme.mlwe_scheme) for _ in range(scheme.mlwe_scheme.r * scheme.ell + scheme.ell)
        ]

    def to_NTT(self) -> None:
        for c in self.obj:
            c.to_NTT()

    def to_coeff(self) -> None:
        for c in self.obj:
            c.to_coeff()

    def _ptrs(self, eng):
        return eng.ffi.new("void*[]", [c.obj for c in self.obj])

    def external_product(self, other: MLWE) -> MLWE:
        res = MLWE(self.scheme.mlwe_scheme)
        self.to_NTT()
        other.to_coeff()
        eng = res.ring.engine
        eng.lib.mgsw_external_product(res.obj, self._ptrs(eng), other.obj, self.scheme.ell,
                                      self.scheme.mlwe_scheme.special_primes)
        eng.check("mgsw_external_product")
        res.repr = repr.ntt
        return res

    def __mul__(self, other):
        if isinstance(other, MLWE):
            return self.external_product(other)
        return NotImplemented


def CMUX(in1: MLWE, in2: MLWE, selector: MGSW) -> MLWE:
    """selector ? in2 : in1 (reference mgsw.py:106-126; mgsw.c:52-72)."""
    res = MLWE(in1.scheme)
    in1.to_coeff()
    in2.to_coeff()
    selector.to_NTT()
    eng = res.ring.engine
    eng.lib.mgsw_CMUX(res.obj, in1.obj, in2.obj, selector._ptrs(eng), selector.scheme.ell, in1.scheme.special_primes)
    eng.check("mgsw_CMUX")
    res.repr = repr.ntt
    return res


class LWE_Key:
    """LWE key with one row per limb (reference lwe.py:18-70)."""

    def __init__(self, ring: Ring, sec_sigma=None, err_sigma=None, sparse_h=None, key=None, n=None):
        self.ring = ring
        self.n = n if n is not None else ring.N
        self.l = ring.ell
        self.q = ring.primes[0]
        lib = ring.lib
        if key is not None:
            self.obj = lib.lwe_alloc_key(self.n, self.l, ring.NTT)
            self.set_s(key)
        elif sparse_h is not None and err_sigma is not None:
            self.obj = lib.lwe_new_sparse_ternary_key(self.n, self.l, ring.NTT, sparse_h, err_sigma)
        elif sec_sigma is not None and err_sigma is not None:
            self.obj = lib.lwe_new_key(self.n, self.l, ring.NTT, sec_sigma, err_sigma)
        else:
            self.obj = lib.lwe_alloc_key(self.n, self.l, ring.NTT)
        ring.engine.check("LWE_Key")

    def set_s(self, key) -> None:
        assert len(key) == self.n
        s = self.ring.ffi.cast("LWE_Key", self.obj).s
        for j in range(self.l):
            q = self.ring.primes[j]
            row = np.frombuffer(self.ring.ffi.buffer(s[j], self.n * 8), dtype=np.uint64)
            row[:] = np.array([int(v) % q for v in key], dtype=np.uint64)

    def set_sigma(self, sigma: float) -> None:
        self.ring.ffi.cast("LWE_Key", self.obj).sigma = sigma

    def get_s(self) -> list[int]:
        s = self.ring.ffi.cast("LWE_Key", self.obj).s
        q0 = self.ring.primes[0]
        row = np.frombuffer(self.ring.ffi.buffer(s[0], self.n * 8), dtype=np.uint64)
        return [int(v) - q0 if int(v) > q0 // 2 else int(v) for v in row]


class LWE:
    """LWE ciphertext with one row per limb (reference lwe.py:73-124)."""

    def __init__(self, ring: Ring, m=None, key: LWE_Key | None = None, is_trivial: bool = False, obj=None, n=None):
        self.ring = ring
        self.n = n if n is not None else ring.N
        self.l = ring.ell
        lib, ffi = ring.lib, ring.ffi
        if obj is not None:
            self.obj = obj
        elif key is not None and m is not None:
            self.n = key.n
            self.obj = lib.lwe_new_sample(ffi.new("uint64_t[]", [x & 0xFFFFFFFFFFFFFFFF for x in m]), key.obj)
        elif is_trivial and m is not None:
            self.obj = lib.lwe_new_trivial_sample(ffi.new("uint64_t[]", [x & 0xFFFFFFFFFFFFFFFF for x in m]),
                                                  self.n, self.l, ring.NTT)
        else:
            self.obj = lib.lwe_alloc_sample(self.n, self.l, ring.NTT)
        ring.engine.check("LWE")

    def __del__(self) -> None:
        with contextlib.suppress(Exception):
            if self.obj is not None:
                self.ring.lib.free_lwe_sample(self.obj)

    def phase(self, key: LWE_Key, recompose: bool = False):
        out = self.ring.ffi.new("uint64_t[]", self.l)
        self.ring.lib.lwe_phase(out, self.obj, key.obj)
        self.ring.engine.check("lwe_phase")
        vals = [int(x) for x in out]
        return crt(vals, self.ring.primes[: self.l]) if recompose else vals

    def subto(self, other: LWE) -> None:
        self.ring.lib.lwe_subto(self.obj, other.obj)
        self.ring.engine.check("lwe_subto")

    def get_a(self) -> list[list[int]]:
        a = self.ring.ffi.cast("LWE", self.obj).a
        return [np.frombuffer(self.ring.ffi.buffer(a[j], self.n * 8), dtype=np.uint64).tolist() for j in range(self.l)]

    def get_b(self) -> list[int]:
        b = self.ring.ffi.cast("LWE", self.obj).b
        return [int(b[j]) for j in range(self.l)]

    def set_rows(self, a: np.ndarray, b) -> None:
        st = self.ring.ffi.cast("LWE", self.obj)
        for j in range(self.l):
            np.frombuffer(self.ring.ffi.buffer(st.a[j], self.n * 8), dtype=np.uint64)[:] = a[j]
            st.b[j] = int(b[j])


def encrypt_lwe(ring: Ring, key_s: list[int], m: list[int], sigma: float, rng: np.random.Generator) -> LWE:
    """Deterministic LWE encryption with host-drawn a and e (lwe.c:95-121 semantics)."""
    n = len(key_s)
    c = LWE(ring, n=n)
    e = int(np.rint(rng.normal(0.0, sigma)))
    a = np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in ring.primes])
    b = []
    for j, q in enumerate(ring.primes):
        s = np.array([v % q for v in key_s], dtype=object)
        acc = int(np.dot(a[j].astype(object), s) % q)
        b.append((acc + e + m[j]) % q)
    c.set_rows(a, b)
    return c

