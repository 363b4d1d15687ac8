"""Batched device API over torch tensors (vfhe_cuda.h Part 2).

Ciphertexts and keys live in HBM as int64 tensors holding uint64 residues:
  ciphertext batch   [B][2][L][N]        (component a, b; limbs in ring order)
  key-switching key  [D][2][L+1][N]      (digit, component, extended limb), NTT domain
Torch supplies device memory and streams only; every operation is one call into the
engine library with raw device pointers.
"""

from __future__ import annotations

import numpy as np
import torch

from .arith import Polynomial, Ring
from .mlwe import MLWE, MLWE_Set
from .native import Engine, EngineError, cuda_engine


def _ptr(ffi, t: torch.Tensor):
    assert t.is_cuda and t.is_contiguous()
    return ffi.cast("uint64_t*", t.data_ptr())


def to_device(a: np.ndarray, device="cuda") -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).to(device)


def to_host(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


class CkksBatch:
    """Batched CKKS evaluation for one level chain of a CKKS scheme."""

    def __init__(self, ring: Ring, special_index: int, engine: Engine | None = None):
        self.engine = engine or cuda_engine()
        self.ring = ring
        self.ffi = self.engine.ffi
        self.lib = self.engine.lib
        self.special = special_index
        self._limbs = self.ffi.new("uint32_t[]", list(ring.prime_indices))
        self.L = ring.ell
        self._ws: torch.Tensor | None = None

    def _stream(self, stream: torch.cuda.Stream | None):
        st = stream or torch.cuda.current_stream()
        return self.ffi.cast("void*", st.cuda_stream)

    def _workspace(self, nbytes: int) -> torch.Tensor:
        if self._ws is None or self._ws.numel() * 8 < nbytes:
            self._ws = torch.empty((nbytes + 7) // 8, dtype=torch.int64, device="cuda")
        return self._ws

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            self.engine.check(what)
            raise EngineError(what)

    def mul_relin_rescale(self, ct1: torch.Tensor, ct2: torch.Tensor, rlk: torch.Tensor,
                          out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        B = ct1.shape[0]
        N = self.ring.N
        if out is None:
            out = torch.empty((B, 2, self.L - 1, N), dtype=torch.int64, device="cuda")
        ws = self._workspace(self.lib.vfhe_cuda_ckks_mul_workspace_bytes(self.ring.NTT, B, self.L))
        rc = self.lib.vfhe_cuda_ckks_mul_relin_rescale_batch(
            self.ring.NTT, _ptr(self.ffi, out), _ptr(self.ffi, ct1), _ptr(self.ffi, ct2), B, self._limbs,
            self.L, self.special, _ptr(self.ffi, rlk), self.ffi.cast("void*", ws.data_ptr()), self._stream(stream))
        self._check(rc, "ckks_mul_relin_rescale_batch")
        return out

    def rotate(self, ct: torch.Tensor, gens: list[int], keys: list[torch.Tensor], out: torch.Tensor | None = None,
               stream=None) -> torch.Tensor:
        B = ct.shape[0]
        if out is None:
            out = torch.empty_like(ct)
        ws = self._workspace(self.lib.vfhe_cuda_ckks_rotate_workspace_bytes(self.ring.NTT, B, self.L))
        g = self.ffi.new("uint64_t[]", [int(x) for x in gens])
        kp = self.ffi.new("uint64_t*[]", [_ptr(self.ffi, k) for k in keys])
        rc = self.lib.vfhe_cuda_ckks_rotate_batch(
            self.ring.NTT, _ptr(self.ffi, out), _ptr(self.ffi, ct), B, self._limbs, self.L, self.special, g, kp,
            self.ffi.cast("void*", ws.data_ptr()), self._stream(stream))
        self._check(rc, "ckks_rotate_batch")
        return out


    def encrypt(self, key, msgs: torch.Tensor | None, batch: int | None = None, sigma: float | None = None,
                out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """Batched encryption under ``key`` (an MLWE_Key of rank 1 at this ring):
        [B][2][L][N] coefficient-domain ciphertexts of the coefficient-domain plaintext
        rows ``msgs`` [B][L][N] (None: ``batch`` encryptions of zero); the batched form
        of CKKS_Scheme.encrypt / mlwe_RNSc_sample (vfhe_cuda_rlwe_encrypt_batch)."""
        B = msgs.shape[0] if msgs is not None else int(batch)
        N = self.ring.N
        if out is None:
            out = torch.empty((B, 2, self.L, N), dtype=torch.int64, device="cuda")
        sk = self._secret_rows(key)
        rc = self.lib.vfhe_cuda_rlwe_encrypt_batch(
            self.ring.NTT, _ptr(self.ffi, out), _ptr(self.ffi, msgs) if msgs is not None else self.ffi.NULL, B,
            self._limbs, self.L, _ptr(self.ffi, sk), float(key.sigma_err if sigma is None else sigma),
            self._stream(stream))
        self._check(rc, "rlwe_encrypt_batch")
        return out

    def _secret_rows(self, key) -> torch.Tensor:
        """The key's secret polynomial at this ring's limbs, NTT domain [L][N] (cached)."""
        cache = getattr(self, "_sk_cache", None)
        if cache is not None and cache[0] is key:
            return cache[1]
        assert len(key.key) == 1, "rank-1 keys only"
        p = Polynomial(self.ring).from_array(key.key[0])
        p.to_NTT()
        sk = to_device(p.rows())
        self._sk_cache = (key, sk)
        return sk


class CggiBatch:
    """Batched CGGI16 functional bootstrap (vfhe_cuda_cggi_bootstrap_batch)."""

    def __init__(self, scheme, engine: Engine | None = None):
        self.engine = engine or cuda_engine()
        self.ffi, self.lib = self.engine.ffi, self.engine.lib
        self.ring = scheme.rings[0]
        self.special = scheme.special_rings[0].prime_indices[-1]
        self._limbs = self.ffi.new("uint32_t[]", list(self.ring.prime_indices))
        self._ws: torch.Tensor | None = None

    def bootstrap(self, lwe_a: torch.Tensor, lwe_b: torch.Tensor, bk: torch.Tensor, tv: torch.Tensor,
                  torus_base: int, stream=None) -> tuple[torch.Tensor, torch.Tensor]:
        B, L0, n = lwe_a.shape
        N = self.ring.N
        out_a = torch.empty((B, L0, N), dtype=torch.int64, device="cuda")
        out_b = torch.empty((B, L0), dtype=torch.int64, device="cuda")
        nbytes = self.lib.vfhe_cuda_cggi_workspace_bytes(self.ring.NTT, B, n, L0)
        if self._ws is None or self._ws.numel() * 8 < nbytes:
            self._ws = torch.empty((nbytes + 7) // 8, dtype=torch.int64, device="cuda")
        st = stream or torch.cuda.current_stream()
        rc = self.lib.vfhe_cuda_cggi_bootstrap_batch(
            self.ring.NTT, _ptr(self.ffi, out_a), _ptr(self.ffi, out_b), _ptr(self.ffi, lwe_a), _ptr(self.ffi, lwe_b),
            B, n, self._limbs, L0, self.special, _ptr(self.ffi, bk), _ptr(self.ffi, tv), torus_base,
            self.ffi.cast("void*", self._ws.data_ptr()), self.ffi.cast("void*", st.cuda_stream))
        if rc != 0:
            self.engine.check("cggi_bootstrap_batch")
            raise EngineError("cggi_bootstrap_batch")
        return out_a, out_b


def gen_ksk_batch(scheme, key_out, polys: list, lvl: int, sigma: float | None = None,
                  engine: Engine | None = None, stream=None) -> torch.Tensor:
    """Key-switching key generated on the GPU (vfhe_cuda_gen_ksk_batch): the batched
    _gen_ksk_components of the scheme (mlwe.py:145-177) for the source polynomials
    ``polys`` at level ``lvl``, as the device tensor [len(polys) * (L+1)][2][L+1][N]
    (NTT domain) that key_tensor() gives for a key generated one digit at a time."""
    engine = engine or cuda_engine()
    ffi, lib = engine.ffi, engine.lib
    sring = scheme.special_rings[lvl]
    P = sring.modulus_ratio(scheme.rings[lvl])
    factors = ffi.new("uint64_t[]", [int(P % q) for q in sring.primes])
    src = []
    for poly in polys:
        if poly.ring != sring:
            poly = Polynomial(sring).from_bigint_array(poly.get_polynomial(signed=True))
        else:
            poly = poly.copy()
        poly.to_NTT()
        src.append(poly.rows())
    d_src = to_device(np.stack(src))
    skp = Polynomial(sring).from_array(key_out.key[0])
    skp.to_NTT()
    d_sk = to_device(skp.rows())
    L, N = sring.ell, sring.N
    out = torch.empty((len(polys) * L, 2, L, N), dtype=torch.int64, device="cuda")
    limbs = ffi.new("uint32_t[]", list(sring.prime_indices))
    st = stream or torch.cuda.current_stream()
    rc = lib.vfhe_cuda_gen_ksk_batch(sring.NTT, _ptr(ffi, out), _ptr(ffi, d_src), len(polys), limbs, L, factors,
                                     _ptr(ffi, d_sk), float(key_out.sigma_err if sigma is None else sigma),
                                     ffi.cast("void*", st.cuda_stream))
    if rc != 0:
        engine.check("gen_ksk_batch")
        raise EngineError("gen_ksk_batch")
    return out


def gen_rlk_batch(scheme, key, lvl: int = 0, **kw) -> torch.Tensor:
    """Relinearisation key (gen_rlk for a rank-1 key) generated on the GPU."""
    return gen_ksk_batch(scheme, key, scheme.quadratic_key_polys(key), lvl, **kw)


def gen_galois_key_batch(scheme, key, gen: int, lvl: int = 0, **kw) -> torch.Tensor:
    """Automorphism key for X -> X^gen (gen_ksk_automorphism) generated on the GPU."""
    return gen_ksk_batch(scheme, key, [p.automorphism(gen) for p in key.poly], lvl, **kw)


def gen_bootstrap_key_batch(cggi, input_key, output_key, sigma: float | None = None, engine: Engine | None = None,
                            stream=None) -> torch.Tensor:
    """RNS CGGI16 bootstrapping key generated on the GPU: the batched
    CGGI16.generate_bootstrap_key (cggi16.py:26-44), i.e. MGSW_Scheme.encrypt
    (mgsw.py:18-55) of every input-key coefficient s_k under the output key, as the
    device tensor [n][2 ell][2][L0+1][N] (NTT domain) that bootstrap_key_tensor() gives
    for a key encrypted one row at a time: rows (0, i) encrypt -s_out s_k (P mod q_i) e_i,
    rows (1, i) encrypt s_k (P mod q_i) e_i.  One vfhe_cuda_gen_ksk_batch call draws all
    of them (it also draws the special prime's digit of each source, whose gadget factor
    is P mod P = 0; those rows are dropped)."""
    from .mlwe import MLWE_Key

    engine = engine or cuda_engine()
    ffi, lib = engine.ffi, engine.lib
    ms = cggi.mgsw_scheme
    scheme = ms.mlwe_scheme
    if scheme.r != 1:
        raise EngineError("gen_bootstrap_key_batch: rank-1 schemes only")
    sring = ms.ring
    lwe_key = input_key.extract_lwe_key() if isinstance(input_key, MLWE_Key) else input_key
    s_in = [int(v) for v in lwe_key.get_s()]
    if any(abs(v) >= 1 << 13 for v in s_in):
        raise EngineError("gen_bootstrap_key_batch: input key coefficients must be small integers")
    n, L, N, ell = len(s_in), sring.ell, sring.N, ms.ell
    P = sring.modulus_ratio(scheme.rings[0])
    factors = ffi.new("uint64_t[]", [int(P % q) for q in sring.primes])
    so = Polynomial(sring).from_array(output_key.key[0])
    so.to_NTT()
    one = Polynomial(sring).from_array([1] + [0] * (N - 1))
    one.to_NTT()
    S, O = so.rows(), one.rows()
    q = np.array(sring.primes, dtype=np.uint64)[:, None]
    src = np.empty((n, 2, L, N), dtype=np.uint64)
    for k, c in enumerate(s_in):
        mag = np.uint64(abs(c))
        ms_k = (S * mag) % q          # |c| s_out, below 2^63 before the reduction
        m_k = (O * mag) % q           # |c| (the NTT of a constant)
        if c > 0:                     # source 0 is -s_out c, source 1 is c
            ms_k = (q - ms_k) % q
        else:
            m_k = (q - m_k) % q
        src[k, 0], src[k, 1] = ms_k, m_k
    d_src = to_device(src.reshape(2 * n, L, N))
    d_sk = to_device(S)
    out = torch.empty((2 * n * L, 2, L, N), dtype=torch.int64, device="cuda")
    limbs = ffi.new("uint32_t[]", list(sring.prime_indices))
    st = stream or torch.cuda.current_stream()
    rc = lib.vfhe_cuda_gen_ksk_batch(sring.NTT, _ptr(ffi, out), _ptr(ffi, d_src), 2 * n, limbs, L, factors,
                                     _ptr(ffi, d_sk), float(output_key.sigma_err if sigma is None else sigma),
                                     ffi.cast("void*", st.cuda_stream))
    if rc != 0:
        engine.check("gen_bootstrap_key_batch")
        raise EngineError("gen_bootstrap_key_batch")
    return out.view(n, 2, L, 2, L, N)[:, :, :ell].reshape(n, 2 * ell, 2, L, N).contiguous()


class WireFormat:
    """Compact host <-> device format of residue rows (vfhe_cuda_pack_rows): each row
    of N residues of a b-bit prime is a bit stream of N b bits, so a ciphertext at the
    CKKS benchmark's chain (one 50-bit and eight 40-bit primes) travels in 46.25 bytes per
    coefficient instead of 72.  ``bits`` lists the width of each row of one item, e.g.
    ``[b_0 .. b_{L-1}] * 2`` for a [2][L][N] ciphertext."""

    def __init__(self, N: int, bits: list[int], engine: Engine | None = None):
        self.engine = engine or cuda_engine()
        self.ffi = self.engine.ffi
        self.lib = self.engine.lib
        self.N = int(N)
        self.bits = [int(b) for b in bits]
        self._bits = self.ffi.new("uint32_t[]", self.bits)
        self.item_bytes = int(self.lib.vfhe_cuda_packed_bytes(self.N, self._bits, len(self.bits), 1))
        if self.item_bytes == 0:
            self.engine.check("packed_bytes")
            raise EngineError("packed_bytes")

    @classmethod
    def for_ring(cls, ring: Ring, components: int = 2, engine: Engine | None = None) -> "WireFormat":
        bits = [int(q).bit_length() for q in ring.primes]
        return cls(ring.N, bits * components, engine)

    def _stream(self, stream):
        st = stream or torch.cuda.current_stream()
        return self.ffi.cast("void*", st.cuda_stream)

    def pack(self, rows: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """[B][rows...][N] int64 residues -> [B][item_bytes] uint8."""
        B = rows.shape[0]
        assert rows.numel() == B * len(self.bits) * self.N and rows.is_contiguous()
        if out is None:
            out = torch.empty((B, self.item_bytes), dtype=torch.uint8, device=rows.device)
        rc = self.lib.vfhe_cuda_pack_rows(self.ffi.cast("void*", out.data_ptr()), _ptr(self.ffi, rows), self.N,
                                          self._bits, len(self.bits), B, self._stream(stream))
        if rc != 0:
            self.engine.check("pack_rows")
            raise EngineError("pack_rows")
        return out

    @staticmethod
    def _host_ptr(ffi, a):
        """Address of a contiguous host array (numpy array or CPU tensor)."""
        if isinstance(a, torch.Tensor):
            assert not a.is_cuda and a.is_contiguous()
            return ffi.cast("void*", a.data_ptr())
        assert a.flags["C_CONTIGUOUS"]
        return ffi.cast("void*", a.ctypes.data)

    def pack_host(self, rows, out=None, nthreads: int = 0):
        """The sender's side on the host (vfhe_cuda_pack_rows_host): [B][rows...][N]
        uint64 / int64 residues in host memory (numpy array or CPU tensor, e.g. pinned)
        -> [B][item_bytes] uint8 in host memory, on `nthreads` threads (0: all)."""
        B = rows.shape[0]
        if out is None:
            out = np.empty((B, self.item_bytes), dtype=np.uint8)
        assert out.shape[0] * out.shape[1] == B * self.item_bytes
        rc = self.lib.vfhe_cuda_pack_rows_host(self._host_ptr(self.ffi, out),
                                               self.ffi.cast("uint64_t*", self._host_ptr(self.ffi, rows)), self.N,
                                               self._bits, len(self.bits), B, int(nthreads))
        if rc != 0:
            self.engine.check("pack_rows_host")
            raise EngineError("pack_rows_host")
        return out

    def unpack_host(self, packed, out, nthreads: int = 0):
        """The receiver's side on the host (vfhe_cuda_unpack_rows_host): [B][item_bytes]
        uint8 -> uint64 / int64 residues in `out` ([B][rows...][N], host memory)."""
        B = packed.shape[0]
        rc = self.lib.vfhe_cuda_unpack_rows_host(self.ffi.cast("uint64_t*", self._host_ptr(self.ffi, out)),
                                                 self._host_ptr(self.ffi, packed), self.N, self._bits,
                                                 len(self.bits), B, int(nthreads))
        if rc != 0:
            self.engine.check("unpack_rows_host")
            raise EngineError("unpack_rows_host")
        return out

    def unpack(self, packed: torch.Tensor, shape: tuple, out: torch.Tensor | None = None,
               stream=None) -> torch.Tensor:
        """[B][item_bytes] uint8 -> int64 residues of ``shape`` ([B][rows...][N])."""
        B = packed.shape[0]
        assert packed.numel() == B * self.item_bytes and packed.is_contiguous()
        if out is None:
            out = torch.empty(shape, dtype=torch.int64, device=packed.device)
        assert out.numel() == B * len(self.bits) * self.N
        rc = self.lib.vfhe_cuda_unpack_rows(_ptr(self.ffi, out), self.ffi.cast("void*", packed.data_ptr()), self.N,
                                            self._bits, len(self.bits), B, self._stream(stream))
        if rc != 0:
            self.engine.check("unpack_rows")
            raise EngineError("unpack_rows")
        return out


def bootstrap_key_tensor(bk) -> torch.Tensor:
    """Device copy of a CGGI16_Key: [n][2 L0][2][L0+1][N] (MGSW rows in encryption order)."""
    arr = np.stack([np.stack([np.stack([c.component_rows(0), c.component_rows(1)]) for c in m.obj]) for m in bk.bk])
    return to_device(arr)


def ciphertext_rows(ct: MLWE) -> np.ndarray:
    """[2][L][N] raw rows of a rank-1 ciphertext."""
    return np.stack([ct.component_rows(0), ct.component_rows(1)])


def key_tensor(ks: MLWE_Set, component: int = 0) -> torch.Tensor:
    """Device copy of one component of a key-switching key set, [D][2][L+1][N]."""
    arr = ks.key_arrays()[component]
    assert arr is not None
    return to_device(arr)
