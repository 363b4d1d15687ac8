"""Complex ring of the CKKS special FFT (reference modules/arith/python/src/vfhe/arith/complex.py).

Buffers are engine-allocated (safe_aligned_malloc, freed with libc free) doubles in the
reference's split layout: n real parts, then n imaginary parts.  The transforms are the
engine's CT_NR / GS_RN / bit_reverse_array / complex_poly_scale_double; on the cuda
engine they run on the GPU with the reference's exact scalar rounding.
"""

from __future__ import annotations

from math import log2

from .arith import Polynomial, Ring, repr
from .native import Engine, default_engine


class ComplexRing:
    """N complex slots with the CKKS special roots (complex.py:21-46)."""

    def __init__(self, N: int, special_rous: bool = True, engine: Engine | None = None):
        self.engine = engine if engine is not None else default_engine()
        self.lib, self.ffi = self.engine.lib, self.engine.ffi
        self.N = N
        self.logN = int(log2(N))
        self.N2 = 2 * N
        self._alloc = self.ffi.new_allocator(alloc=lambda size: self.lib.safe_aligned_malloc(size),
                                             free=lambda ptr: self.lib.free(ptr), should_clear_after_alloc=True)
        if special_rous:
            rous = self.gen_special_rous_hp(self.N2)
            self.CT_rous = self.lib.load_rous_CT(self.ffi.new("double[]", [r.real for r in rous]),
                                                 self.ffi.new("double[]", [r.imag for r in rous]), self.N2)
            inv = [r**-1 for r in rous]
            self.GS_rous = self.lib.load_rous_GS(self.ffi.new("double[]", [r.real for r in inv]),
                                                 self.ffi.new("double[]", [r.imag for r in inv]), self.N2)
            self.engine.check("load_rous")

    def alloc_polynomial(self):
        return self._alloc("double[]", self.N2)

    def exp_complex_polys_ifft_scale_round_to_RNS_batch(self, e_polys: list["ComplexPolynomial"], ring: Ring,
                                                        temp_delta: float) -> list[Polynomial]:
        """For each slot-domain polynomial: IFFT, scale by temp_delta, round to RNS (NTT domain)
        (complex.py:48-73)."""
        n = len(e_polys)
        if n == 0:
            return []
        res = [Polynomial(ring) for _ in range(n)]
        rows = self.ffi.new("void*[]", [self.ffi.cast("void *", p.obj) for p in e_polys])
        outs = self.ffi.new("void*[]", [self.ffi.cast("void *", p.obj) for p in res])
        self.lib.complex_polys_ifft_scale_round_to_RNS_batch(rows, outs, n, self.N, self.logN, self.GS_rous,
                                                             temp_delta)
        self.engine.check("complex_polys_ifft_scale_round_to_RNS_batch")
        for p in res:
            p.repr = repr.ntt
        return res

    @staticmethod
    def gen_special_rous_hp(N: int) -> list[complex]:
        """Entry 2^(k-1)+i = w^((5^brv(i)) N / 2^(k+1)), w = exp(2 pi i / 2N), 100-bit
        mpmath rounded to complex128 (complex.py:90-106)."""
        import mpmath as mp

        N = int(N)
        mp.mp.prec = 100
        rou = mp.exp(2 * mp.pi * 1j / (2 * mp.mpf(N)))

        def brev(x, size):
            return int(bin(x)[2:].rjust(size, "0")[::-1], 2)

        result = [1] * N
        for k in range(int(log2(N)) - 1, 0, -1):
            for i in range(2 ** (k - 1)):
                expo = ((5 ** brev(i, k - 1)) * N // (2 ** (k + 1))) % (2 * N)
                result[2 ** (k - 1) + i] = mp.power(rou, expo)
        return [complex(i) for i in result]


class ComplexPolynomial:
    """(complex.py:109-162)"""

    def __init__(self, ring: ComplexRing):
        self.ring = ring
        self.obj = ring.alloc_polynomial()

    def __iter__(self):
        n = self.ring.N
        return iter([self.obj[i] + self.obj[i + n] * 1j for i in range(n)])

    def __getitem__(self, i: int) -> complex:
        return self.obj[i] + self.obj[i + self.ring.N] * 1j

    def __setitem__(self, i: int, v: complex) -> None:
        v = complex(v)
        self.obj[i] = v.real
        self.obj[i + self.ring.N] = v.imag

    def from_array(self, values) -> "ComplexPolynomial":
        n = self.ring.N
        for i, v in enumerate(values):
            v = complex(v)
            self.obj[i] = v.real
            self.obj[i + n] = v.imag
        return self

    def IFFT(self) -> None:
        lib = self.ring.lib
        lib.bit_reverse_array(self.obj, self.ring.N, self.ring.logN)
        lib.GS_RN(self.obj, self.ring.GS_rous, self.ring.N)
        lib.complex_poly_scale_double(self.obj, 1.0 / self.ring.N, self.ring.N)
        self.ring.engine.check("ComplexPolynomial.IFFT")

    def FFT(self) -> None:
        lib = self.ring.lib
        lib.CT_NR(self.obj, self.ring.CT_rous, self.ring.N)
        lib.bit_reverse_array(self.obj, self.ring.N, self.ring.logN)
        self.ring.engine.check("ComplexPolynomial.FFT")

    def __imul__(self, other):
        if isinstance(other, (int, float)):
            self.ring.lib.complex_poly_scale_double(self.obj, float(other), self.ring.N)
            self.ring.engine.check("complex_poly_scale_double")
            return self
        raise NotImplementedError(f"cannot scale by {type(other).__name__}")

    def round_to_RNS_cpp(self, ring: Ring) -> Polynomial:
        res = Polynomial(ring)
        self.ring.lib.complex_poly_round_to_RNS(res.obj, self.obj, ring.N)
        self.ring.engine.check("complex_poly_round_to_RNS")
        res.repr = repr.ntt
        return res
