"""RNS rings and polynomials over an engine library.

Host-side mirror of the reference's ``vfhe.arith`` operator surface
(modules/arith/python/src/vfhe/arith/polynomial.py, ntt.py): the same class and
method names and argument meaning, so code written against the reference reads the
same here.  Every arithmetic method is one call into the engine (the cuda library by
default); bulk coefficient IO goes through numpy views of the engine's rows instead
of per-element cffi accesses.
"""

from __future__ import annotations

import contextlib
import math
from enum import Enum

import numpy as np

from .native import Engine, default_engine
from .numbers import crt, is_prime


def next_power_of_2(x: float) -> int:
    return 1 << math.ceil(math.log2(x))


class NTTProcessor:
    """Per-engine pool of primes for each (N, split_degree) (reference ntt.py:10-62).

    A pool is one ``incNTT``; rings sharing (N, split_degree) share it, and a ring's
    limbs are its primes' indices in the pool.
    """

    def __init__(self, engine: Engine):
        self.engine = engine
        self.incNTTs: dict[tuple[int, int], object] = {}
        self.primes: dict[tuple[int, int], list[int]] = {}
        self.prime_to_index: dict[tuple[int, int], dict[int, int]] = {}
        self.conversion_params_cache: dict[tuple, object] = {}

    def register_ring_primes(self, primes: list[int], N: int, split_degree: int) -> list[int]:
        ffi, lib = self.engine.ffi, self.engine.lib
        key = (N, split_degree)
        if key not in self.incNTTs:
            handle = lib.new_incomplete_ntt_list(ffi.new("uint64_t[]", list(primes)), split_degree, N, len(primes))
            self.engine.check("new_incomplete_ntt_list")
            if handle == ffi.NULL:
                raise RuntimeError("new_incomplete_ntt_list failed")
            self.incNTTs[key] = handle
            self.primes[key] = list(primes)
            self.prime_to_index[key] = {p: i for i, p in enumerate(primes)}
        else:
            pmap = self.prime_to_index[key]
            new = [p for p in primes if p not in pmap]
            if new:
                start = len(self.primes[key])
                lib.incNTT_extend_with_primes(self.incNTTs[key], ffi.new("uint64_t[]", new), len(new))
                self.engine.check("incNTT_extend_with_primes")
                for i, p in enumerate(new):
                    self.primes[key].append(p)
                    pmap[p] = start + i
        return [self.prime_to_index[key][p] for p in primes]

    def get_conversion_params(self, N: int, split_degree: int, in_mask: int, out_mask: int):
        key = (N, split_degree, in_mask, out_mask, tuple(self.primes[(N, split_degree)]))
        if key not in self.conversion_params_cache:
            params = self.engine.lib.init_base_conversion_params(self.incNTTs[(N, split_degree)], in_mask, out_mask)
            self.engine.check("init_base_conversion_params")
            self.conversion_params_cache[key] = params
        return self.conversion_params_cache[key]

    def reset(self) -> None:
        self.incNTTs.clear()
        self.primes.clear()
        self.prime_to_index.clear()
        self.conversion_params_cache.clear()


_PROCESSORS: dict[int, NTTProcessor] = {}


def ntt_processor(engine: Engine) -> NTTProcessor:
    proc = _PROCESSORS.get(id(engine))
    if proc is None or proc.engine is not engine:
        proc = NTTProcessor(engine)
        _PROCESSORS[id(engine)] = proc
    return proc


def reset_registries() -> None:
    """Forget every prime pool (the reference's tests do this per test, conftest.py:63-85)."""
    for p in _PROCESSORS.values():
        p.reset()


class Ring:
    """Z_Q[X]/(X^N+1) in RNS form (reference polynomial.py:20-187)."""

    def __init__(
        self,
        N: int,
        mod_size: int | None = None,
        split_degree: int | None = None,
        primes: list[int] | None = None,
        mask: int | None = None,
        prime_size: int | list[int] = 49,
        exceptional_set_size: int = 128,
        engine: Engine | None = None,
    ) -> None:
        assert (
            mod_size is not None or isinstance(prime_size, list) or primes is not None or mask is not None
        ), "must provide mod_size, prime_size, primes, or mask"
        self.engine = engine if engine is not None else default_engine()
        self.lib = self.engine.lib
        self.ffi = self.engine.ffi
        proc = ntt_processor(self.engine)

        if mask is not None:
            assert primes is not None, "must provide primes when mask is given"
            split = split_degree
            if not split:
                smallest = min(math.ceil(math.log2(p)) for p in primes)
                split = next_power_of_2(exceptional_set_size / smallest)
            pmap = proc.prime_to_index[(N, split)]
            primes = [p for p in primes if (mask >> pmap[p]) & 1]
            prime_size = [math.ceil(math.log2(p)) for p in primes]

        if primes is not None and prime_size is None:
            prime_size = [math.ceil(math.log2(p)) for p in primes]

        if isinstance(prime_size, list):
            self.ell = len(prime_size)
            self.prime_size = list(prime_size)
            self.smallest_prime = min(prime_size)
        else:
            self.ell = math.ceil(mod_size / prime_size)  # type: ignore[operator]
            self.prime_size = [prime_size] * self.ell
            self.smallest_prime = prime_size

        if not split_degree:
            split_degree = next_power_of_2(exceptional_set_size / self.smallest_prime)
        self.split_degree = split_degree
        self.N = N
        self.byte_size = N * self.ell * 8

        if primes:
            assert len(primes) >= self.ell, "not enough primes"
            self.primes = list(primes[: self.ell])
        else:
            self.primes = self.gen_primes()
        self.q_l = math.prod(self.primes)
        self.bit_size = math.ceil(math.log2(self.q_l))
        self.prime_indices = proc.register_ring_primes(self.primes, N, split_degree)
        self.NTT = proc.incNTTs[(N, split_degree)]
        self.mask = sum(1 << i for i in self.prime_indices)

    # -- pool views
    def _ntt_l(self) -> int:
        return int(self.ffi.cast("incNTT", self.NTT).l)

    def get_rou_matrix(self) -> list[list[int]]:
        w = self.lib.incNTT_get_rou_matrix(self.NTT)
        P = self.N // self.split_degree
        return [np.frombuffer(self.ffi.buffer(w[i], P * 8), dtype=np.uint64).tolist() for i in self.prime_indices]

    # -- ring relations
    def quotient_ring(self, mod_size=None, ell=None, mask=None) -> Ring:
        assert (mod_size is not None) ^ (ell is not None) ^ (mask is not None)
        if mod_size is not None:
            return Ring(self.N, mod_size, self.split_degree, primes=self.primes, engine=self.engine)
        if ell is not None:
            return Ring(self.N, prime_size=self.prime_size[:ell], split_degree=self.split_degree,
                        primes=self.primes, engine=self.engine)
        return Ring(self.N, mask=mask, split_degree=self.split_degree, primes=self.primes, engine=self.engine)

    def is_quotient_ring(self, parent: Ring) -> bool:
        return parent.mask & self.mask == self.mask

    def modulus_ratio(self, other: Ring, return_pointer: bool = False):
        assert other.is_quotient_ring(self), "other_ring must be a quotient ring of this ring"
        scaling = self.mask & ~other.mask
        delta = math.prod(p for p, idx in zip(self.primes, self.prime_indices) if (scaling >> idx) & 1)
        if return_pointer:
            arr = [0] * self._ntt_l()
            for p, idx in zip(self.primes, self.prime_indices):
                arr[idx] = delta % p
            return self.ffi.new("uint64_t[]", arr)
        return delta

    def intersec(self, other: Ring) -> Ring:
        if self == other:
            return self
        if self.ell > other.ell:
            assert other.is_quotient_ring(self)
            return other
        assert self.is_quotient_ring(other)
        return self

    # -- primes (reference polynomial.py:151-170): the largest primes 1 mod rou_order
    #    below 2^prime_size, searched downwards over odd multiples
    @staticmethod
    def gen_prime(rou_order: int, prime_size: int, exclude_list=None) -> int:
        exclude = set(exclude_list or [])
        a = (((1 << prime_size) - 1) // rou_order) | 1
        a -= 2
        while True:
            cand = a * rou_order + 1
            if cand not in exclude and is_prime(cand):
                return cand
            a -= 2

    def gen_primes(self) -> list[int]:
        primes: list[int] = []
        for size in self.prime_size:
            primes.append(Ring.gen_prime(2 * self.N // self.split_degree, size, exclude_list=primes))
        return primes

    def alloc_polynomial(self):
        h = self.lib.polynomial_new_RNS_polynomial(self.N, self.mask, self.NTT)
        self.engine.check("polynomial_new_RNS_polynomial")
        return h

    def scalar_array(self, value):
        arr = [0] * self._ntt_l()
        if isinstance(value, int):
            for p, idx in zip(self.primes, self.prime_indices):
                arr[idx] = value % p
        else:
            vals = list(value)
            assert len(vals) == self.ell
            for v, idx in zip(vals, self.prime_indices):
                arr[idx] = v
        return self.ffi.new("uint64_t[]", arr)

    def random_element(self, ntt: bool = True) -> Polynomial:
        return Polynomial(self).sample_uniform(ntt)

    def random_gaussian_element(self, sigma: float, ntt: bool = True) -> Polynomial:
        return Polynomial(self).sample_gaussian(sigma, ntt)

    def random_exceptional(self, size="minimal", ntt: bool = True) -> Polynomial:
        return Polynomial(self).sample_exceptional(size, ntt)

    # -- layout helpers: coefficient j sits at row position (j mod s) * P + j // s
    def layout_perm(self) -> np.ndarray:
        s = self.split_degree
        P = self.N // s
        j = np.arange(self.N)
        return (j % s) * P + j // s

    def __repr__(self) -> str:
        return f"Ring(N={self.N}, primes={self.primes}, split={self.split_degree}, mask={self.mask:#x})"


repr = Enum("Polynomial Representation", ["empty", "ntt", "coeff"])  # noqa: A001


class Polynomial:
    """An RNS polynomial handle (reference polynomial.py:195-634)."""

    def __init__(self, ring: Ring, repr=repr.empty) -> None:  # noqa: A002
        self.ring = ring
        self.obj = ring.alloc_polynomial()
        self.repr = repr

    # -- engine plumbing
    @property
    def _lib(self):
        return self.ring.lib

    def _chk(self, what: str) -> None:
        self.ring.engine.check(what)

    @property
    def rns_mask(self) -> int:
        return int(self.ring.ffi.cast("RNS_Polynomial", self.obj).rns_mask)

    @rns_mask.setter
    def rns_mask(self, value: int) -> None:
        self.ring.ffi.cast("RNS_Polynomial", self.obj).rns_mask = value

    def row(self, idx: int) -> np.ndarray:
        """Writable numpy view of pool row ``idx`` (N residues)."""
        p = self.ring.ffi.cast("RNS_Polynomial", self.obj)
        return np.frombuffer(self.ring.ffi.buffer(p.coeffs[idx], self.ring.N * 8), dtype=np.uint64)

    def __del__(self) -> None:
        with contextlib.suppress(Exception):
            self.ring.lib.free_RNS_polynomial(self.obj)

    # -- construction
    def from_array(self, array) -> Polynomial:
        vals = list(array) + [0] * (self.ring.N - len(array))
        buf = np.array([int(x) & 0xFFFFFFFFFFFFFFFF for x in vals], dtype=np.uint64)
        self._lib.int_array_to_RNS(self.obj, self.ring.ffi.from_buffer("uint64_t[]", buf))
        self._chk("int_array_to_RNS")
        self.repr = repr.ntt
        return self

    def from_bigint_array(self, array) -> Polynomial:
        ffi = self.ring.ffi
        rows = [ffi.NULL] * self.ring._ntt_l()
        keep = []
        for p, idx in zip(self.ring.primes, self.ring.prime_indices):
            buf = np.array([int(v) % p for v in array], dtype=np.uint64)
            keep.append(buf)
            rows[idx] = ffi.from_buffer("uint64_t[]", buf)
        self._lib.array_to_RNS(self.obj, ffi.new("uint64_t*[]", rows))
        self._chk("array_to_RNS")
        self.repr = repr.ntt
        return self

    def fast_inverse(self) -> Polynomial:
        assert self.repr == repr.ntt
        out = Polynomial(self.ring)
        rc = self._lib.polynomial_RNS_inverse(out.obj, self.obj)
        if rc == -2:
            raise ValueError("polynomial_RNS_inverse: zero slot is not invertible")
        self._chk("polynomial_RNS_inverse")
        if rc != 0:
            raise RuntimeError(f"polynomial_RNS_inverse failed with code {rc}")
        out.repr = repr.ntt
        return out

    # -- arithmetic (in place on self)
    def multiply(self, in1: Polynomial, in2: Polynomial) -> None:
        assert in1.repr == in2.repr == repr.ntt
        self._lib.polynomial_mul_RNS_polynomial(self.obj, in1.obj, in2.obj)
        self._chk("polynomial_mul_RNS_polynomial")
        self.repr = in1.repr

    def negate(self, in1: Polynomial | None = None) -> None:
        in1 = in1 or self
        self._lib.polynomial_RNSc_negate(self.obj, in1.obj)
        self._chk("polynomial_RNSc_negate")
        self.repr = in1.repr

    def sub(self, in1: Polynomial, in2: Polynomial) -> None:
        assert in1.repr == in2.repr
        f = self._lib.polynomial_sub_RNS_polynomial if in1.repr == repr.ntt else self._lib.polynomial_sub_RNSc_polynomial
        f(self.obj, in1.obj, in2.obj)
        self._chk("polynomial_sub")
        self.repr = in1.repr

    def add(self, in1: Polynomial, in2: Polynomial) -> None:
        assert in1.repr == in2.repr
        f = self._lib.polynomial_add_RNS_polynomial if in1.repr == repr.ntt else self._lib.polynomial_add_RNSc_polynomial
        f(self.obj, in1.obj, in2.obj)
        self._chk("polynomial_add")
        self.repr = in1.repr

    def automorphism(self, gen: int) -> Polynomial:
        assert gen < self.ring.N * 2
        res = Polynomial(self.ring)
        self.to_coeff()
        self._lib.polynomial_RNSc_permute(res.obj, self.obj, gen)
        self._chk("polynomial_RNSc_permute")
        res.repr = repr.coeff
        return res

    def to_NTT(self) -> None:
        if self.repr == repr.ntt:
            return
        self._lib.polynomial_RNSc_to_RNS(self.obj, self.obj)
        self._chk("polynomial_RNSc_to_RNS")
        self.repr = repr.ntt

    def to_coeff(self) -> None:
        if self.repr == repr.coeff:
            return
        self._lib.polynomial_RNS_to_RNSc(self.obj, self.obj)
        self._chk("polynomial_RNS_to_RNSc")
        self.repr = repr.coeff

    def to_repr(self, r) -> None:
        if r == repr.ntt:
            self.to_NTT()
        if r == repr.coeff:
            self.to_coeff()

    # -- sampling (engine random stream)
    def sample_uniform(self, ntt: bool = True) -> Polynomial:
        self._lib.polynomial_gen_random_RNSc_polynomial(self.obj)
        self._chk("polynomial_gen_random_RNSc_polynomial")
        self.repr = repr.ntt if ntt else repr.coeff
        return self

    def sample_gaussian(self, sigma: float, ntt: bool = True) -> Polynomial:
        self._lib.polynomial_gen_gaussian_RNSc_polynomial(self.obj, sigma)
        self._chk("polynomial_gen_gaussian_RNSc_polynomial")
        self.repr = repr.coeff
        if ntt:
            self.to_NTT()
        return self

    def sample_exceptional(self, size="minimal", ntt: bool = True) -> Polynomial:
        self._lib.polynomial_gen_random_RNSc_polynomial(self.obj)
        self._lib.polynomial_RNS_broadcast_slot(self.obj, self.obj, 0)
        self._chk("sample_exceptional")
        self.repr = repr.ntt
        if not ntt:
            self.to_coeff()
        return self

    # -- tower
    def base_extend(self, ring: Ring | None = None, out: Polynomial | None = None) -> Polynomial:
        out_ = out if out is not None else Polynomial(ring)  # type: ignore[arg-type]
        assert self.ring.is_quotient_ring(out_.ring), "Not a quotient ring"
        return self.lift_to(out=out_)

    def lift_to(self, ring: Ring | None = None, out: Polynomial | None = None, params=None) -> Polynomial:
        self.to_coeff()
        out_ = out if out is not None else Polynomial(ring)  # type: ignore[arg-type]
        if params is None:
            params = ntt_processor(self.ring.engine).get_conversion_params(
                self.ring.N, self.ring.split_degree, self.rns_mask, out_.rns_mask
            )
        self._lib.polynomial_base_conversion_RNSc(out_.obj, self.obj, params)
        self._chk("polynomial_base_conversion_RNSc")
        out_.repr = repr.coeff
        return out_

    def mod_reduce(self, ring: Ring | None = None, out: Polynomial | None = None) -> Polynomial:
        self.to_coeff()
        out_ = out if out is not None else Polynomial(ring)  # type: ignore[arg-type]
        assert out_.ring.is_quotient_ring(self.ring), "Not a quotient ring"
        self._lib.polynomial_RNSc_mod_reduce(out_.obj, self.obj)
        self._chk("polynomial_RNSc_mod_reduce")
        out_.repr = repr.coeff
        return out_

    def floor_division(self, ring: Ring) -> Polynomial:
        assert ring.ell < self.ring.ell and ring.is_quotient_ring(self.ring)
        self.to_coeff()
        self._lib.polynomial_floor_division_RNSc_wo_free(self.obj, self.rns_mask & ~ring.mask)
        self._chk("polynomial_floor_division_RNSc_wo_free")
        self.ring = ring
        return self

    def round_division(self, ring: Ring) -> Polynomial:
        assert ring.ell < self.ring.ell and ring.is_quotient_ring(self.ring)
        self.to_coeff()
        self._lib.polynomial_round_division_RNSc_wo_free(self.obj, self.rns_mask & ~ring.mask)
        self._chk("polynomial_round_division_RNSc_wo_free")
        self.ring = ring
        return self

    def scaled_lift(self, ring: Ring, delta=None) -> Polynomial:
        self.to_coeff()
        out = Polynomial(ring)
        self._lib.polynomial_RNSc_scaled_lift(out.obj, self.obj, delta if delta is not None else self.ring.ffi.NULL)
        self._chk("polynomial_RNSc_scaled_lift")
        out.repr = repr.coeff
        return out

    # -- coefficient IO
    def rows(self) -> np.ndarray:
        """Raw rows of the ring's limbs, [ell][N] uint64, in the engine's row layout."""
        return np.stack([self.row(i).copy() for i in self.ring.prime_indices])

    def set_rows(self, rows: np.ndarray) -> None:
        for k, idx in enumerate(self.ring.prime_indices):
            self.row(idx)[:] = np.asarray(rows[k], dtype=np.uint64)

    def coeff_array(self, r=None) -> np.ndarray:
        """[ell][N] residues in natural coefficient order (numpy)."""
        r = repr.coeff if r is None else r
        if self.repr != r:
            self.to_repr(r)
        return self.rows()[:, self.ring.layout_perm()]

    def get_coeff_matrix(self, repr=repr.coeff) -> list[list[int]]:  # noqa: A002
        return self.coeff_array(repr).tolist()

    def from_coeff_matrix(self, matrix, repr=repr.coeff) -> Polynomial:  # noqa: A002
        perm = self.ring.layout_perm()
        for k, idx in enumerate(self.ring.prime_indices):
            dst = self.row(idx)
            dst[perm] = np.asarray([int(v) for v in matrix[k]] if not isinstance(matrix[k], np.ndarray)
                                   else matrix[k], dtype=np.uint64)
        self.repr = repr
        return self

    def get_polynomial(self, signed: bool = False) -> list[int]:
        self.to_coeff()
        rns = self.coeff_array()
        if self.ring.ell == 1:
            vals = [int(x) for x in rns[0]]
        else:
            vals = [crt([int(rns[i][j]) for i in range(self.ring.ell)], self.ring.primes) for j in range(self.ring.N)]
        if not signed:
            return vals
        q = self.ring.q_l
        return [min(v, -(q - v), key=abs) for v in vals]

    def __eq__(self, value) -> bool:  # type: ignore[override]
        if isinstance(value, int):
            m = self.coeff_array()
            return bool(np.all(m[:, 0] == value) and np.all(m[:, 1:] == 0))
        if isinstance(value, list):
            m = self.coeff_array()
            return all(int(m[i][0]) == value[i] and not m[i][1:].any() for i in range(self.ring.ell))
        self.to_repr(value.repr)
        res = bool(self._lib.polynomial_eq(self.obj, value.obj))
        self._chk("polynomial_eq")
        return res

    __hash__ = None  # type: ignore[assignment]

    def __repr__(self) -> str:
        return str(self.get_coeff_matrix())

    def __iter__(self):
        return iter(self.get_coeff_matrix())

    def copy(self) -> Polynomial:
        res = Polynomial(self.ring)
        self._lib.polynomial_copy_RNS_polynomial(res.obj, self.obj)
        self._chk("polynomial_copy_RNS_polynomial")
        res.repr = self.repr
        return res

    __copy__ = copy

    def __mod__(self, value: int) -> Polynomial:
        self.to_coeff()
        res = Polynomial(self.ring)
        self._lib.polynomial_RNSc_mod_reduce_lifted(res.obj, self.obj, self.ring.primes.index(value))
        self._chk("polynomial_RNSc_mod_reduce_lifted")
        return res

    def __itruediv__(self, value: int) -> Polynomial:
        self.to_coeff()
        self._lib.polynomial_round_division_RNSc_wo_free(self.obj, 1 << self.ring.primes.index(value))
        self._chk("polynomial_round_division_RNSc_wo_free")
        return self

    def __mul__(self, other):
        if isinstance(other, Polynomial):
            self.to_NTT()
            other.to_NTT()
            res = Polynomial(self.ring.intersec(other.ring))
            res.multiply(self, other)
            return res
        if isinstance(other, int):
            if other == 0:
                return 0
            if other == 1:
                return self.copy()
            res = Polynomial(self.ring)
            self._lib.polynomial_scale_RNSc_polynomial(res.obj, self.obj, other % (1 << 64))
            self._chk("polynomial_scale_RNSc_polynomial")
            res.repr = self.repr
            return res
        if isinstance(other, list):
            res = Polynomial(self.ring)
            assert len(other) == self.ring.ell
            self._lib.polynomial_scale_RNS_polynomial_RNS(res.obj, self.obj, self.ring.scalar_array(other))
            self._chk("polynomial_scale_RNS_polynomial_RNS")
            res.repr = self.repr
            return res
        raise NotImplementedError(f"cannot multiply by {type(other).__name__}")

    def __rmul__(self, other):
        return self.__mul__(other)

    def __imul__(self, other):
        if isinstance(other, Polynomial):
            self.to_NTT()
            other.to_NTT()
            self._lib.polynomial_multo_RNS_polynomial(self.obj, other.obj)
            self._chk("polynomial_multo_RNS_polynomial")
        elif isinstance(other, int):
            if other == 0:
                return 0
            if other == 1:
                return self
            self._lib.polynomial_scale_RNSc_polynomial(self.obj, self.obj, other)
            self._chk("polynomial_scale_RNSc_polynomial")
        else:
            raise NotImplementedError
        return self

    def __add__(self, other):
        if isinstance(other, int):
            if other == 0:
                return self.copy()
            res = Polynomial(self.ring)
            f = self._lib.polynomial_RNSc_add_integer if self.repr == repr.coeff else self._lib.polynomial_RNS_add_integer
            f(res.obj, self.obj, other & 0xFFFFFFFFFFFFFFFF)
            self._chk("add_integer")
            res.repr = self.repr
            return res
        if self.repr != other.repr:
            self.to_NTT()
            other.to_NTT()
        res = Polynomial(self.ring.intersec(other.ring))
        res.add(self, other)
        return res

    def __radd__(self, other):
        return self.__add__(other)

    def __iadd__(self, other):
        if isinstance(other, int):
            if other == 0:
                return self
            raise NotImplementedError("nonzero int operand not supported")
        if not isinstance(other, Polynomial):
            return other + self
        if self.repr != other.repr:
            self.to_NTT()
            other.to_NTT()
        self.add(self, other)
        return self

    def __isub__(self, other):
        if isinstance(other, int):
            if other == 0:
                return self
            raise NotImplementedError("nonzero int operand not supported")
        if self.repr != other.repr:
            self.to_NTT()
            other.to_NTT()
        self.sub(self, other)
        return self

    def __neg__(self) -> Polynomial:
        res = Polynomial(self.ring)
        res.negate(self)
        return res

    def __sub__(self, other):
        if isinstance(other, int):
            if other == 0:
                return self.copy()
            raise NotImplementedError("nonzero int operand not supported")
        if self.repr != other.repr:
            self.to_NTT()
            other.to_NTT()
        res = Polynomial(self.ring.intersec(other.ring))
        res.sub(self, other)
        return res

    def __rsub__(self, other):
        return (-self) + other
