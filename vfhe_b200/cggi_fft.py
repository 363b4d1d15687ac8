"""CGGI over the 32-bit torus with FP64 FFT external products (vfhe_cuda_cggi_fft_*).

Host side: parameters, seeded key generation and encryption (numpy; exact integer
arithmetic through float64 matrix products whose sums stay below 2^53), the lookup
test vector and decryption.  Device side: :class:`CggiFft` keeps the bootstrapping
key's spectra and the key-switching key in HBM and runs the batched programmable
bootstrap (one persistent blind-rotation launch + one key-switch launch).

The default parameters are the classic TFHE set: LWE n = 630 with a binary key and
sigma = 2^-15; GLWE N = 1024, k = 1, binary key, sigma = 2^-25; bootstrapping gadget
base 2^7 with 3 levels; key switching base 2^2 with 8 levels.  Messages carry 4 bits
plus a padding bit (delta = 2^27); the lookup table has 16 entries.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .native import Engine, EngineError, cuda_engine

MASK32 = (1 << 32) - 1


@dataclass(frozen=True)
class TorusParams:
    n: int = 630
    N: int = 1024
    lwe_sigma: float = 2.0**-15
    glwe_sigma: float = 2.0**-25
    bs_base_log: int = 7
    bs_levels: int = 3
    ks_base_log: int = 2
    ks_levels: int = 8
    msg_bits: int = 4

    @property
    def t(self) -> int:  # lookup-table size
        return 1 << self.msg_bits

    @property
    def delta(self) -> int:  # message scale, one padding bit above the message
        return 1 << (32 - self.msg_bits - 1)


def _noise(rng: np.random.Generator, sigma: float, shape) -> np.ndarray:
    return np.rint(rng.normal(0.0, sigma * 2.0**32, shape)).astype(np.int64)


def _u32(x: np.ndarray) -> np.ndarray:
    return (np.asarray(x, dtype=np.int64) & MASK32).astype(np.uint32)


def negacyclic_times_binary(A: np.ndarray, S: np.ndarray) -> np.ndarray:
    """A [..., N] torus rows times a binary polynomial S, mod (X^N + 1, 2^32), exact:
    a float64 matrix product of integers whose sums stay below 2^53."""
    N = S.shape[0]
    idx = (np.arange(N)[:, None] - np.arange(N)[None, :])  # i - j
    C = np.where(idx >= 0, S[idx % N], -S[idx % N]).astype(np.float64)  # out_i = sum_j a_j C[i, j]
    flat = A.reshape(-1, N).astype(np.float64)
    out = flat @ C.T
    return _u32(np.mod(out, 2.0**32).astype(np.int64)).reshape(A.shape)


def lwe_dot(A: np.ndarray, s: np.ndarray) -> np.ndarray:
    """<a, s> mod 2^32 for rows of A (torus) and a small integer key s, exact."""
    hi = (A.astype(np.int64) >> 16).astype(np.float64) @ s.astype(np.float64)
    lo = (A.astype(np.int64) & 0xFFFF).astype(np.float64) @ s.astype(np.float64)
    return _u32((np.mod(hi, 2.0**16).astype(np.int64) << 16) + lo.astype(np.int64))


@dataclass
class TorusKeys:
    params: TorusParams
    s: np.ndarray    # LWE key, int32 [n], binary
    S: np.ndarray    # GLWE key, int32 [N], binary
    bsk: np.ndarray  # uint32 [n][2 levels][2][N]: GGSW(s_i), row (c, l) at c * levels + l
    ksk: np.ndarray  # uint32 [N][ks_levels][n + 1]: LWE_s(S_j 2^(32 - kb (l + 1)))

    @staticmethod
    def generate(params: TorusParams, rng: np.random.Generator) -> "TorusKeys":
        p = params
        s = rng.integers(0, 2, p.n).astype(np.int32)
        S = rng.integers(0, 2, p.N).astype(np.int32)
        R = 2 * p.bs_levels
        a = rng.integers(0, 1 << 32, (p.n, R, p.N), dtype=np.uint64).astype(np.uint32)
        b = negacyclic_times_binary(a, S).astype(np.int64) + _noise(rng, p.glwe_sigma, (p.n, R, p.N))
        bsk = np.zeros((p.n, R, 2, p.N), dtype=np.int64)
        bsk[:, :, 0] = a
        bsk[:, :, 1] = b
        for c in range(2):
            for lv in range(p.bs_levels):
                bsk[:, c * p.bs_levels + lv, c, 0] += s.astype(np.int64) << (32 - p.bs_base_log * (lv + 1))
        ka = rng.integers(0, 1 << 32, (p.N, p.ks_levels, p.n), dtype=np.uint64).astype(np.uint32)
        kb = lwe_dot(ka.reshape(-1, p.n), s).reshape(p.N, p.ks_levels).astype(np.int64)
        kb += _noise(rng, p.lwe_sigma, (p.N, p.ks_levels))
        kb += S[:, None].astype(np.int64) << (32 - p.ks_base_log * (np.arange(p.ks_levels)[None, :] + 1))
        ksk = np.concatenate([ka, _u32(kb)[..., None]], axis=2)
        return TorusKeys(p, s, S, _u32(bsk), ksk)

    def encrypt(self, messages, rng: np.random.Generator) -> np.ndarray:
        """LWE encryptions [B][n+1] of messages m in [0, t) at m * delta."""
        p = self.params
        m = np.asarray(messages, dtype=np.int64)
        A = rng.integers(0, 1 << 32, (len(m), p.n), dtype=np.uint64).astype(np.uint32)
        b = lwe_dot(A, self.s).astype(np.int64) + _noise(rng, p.lwe_sigma, len(m)) + m * p.delta
        return np.concatenate([A, _u32(b)[:, None]], axis=1)

    def phases(self, lwe: np.ndarray, key: np.ndarray | None = None) -> np.ndarray:
        """Signed torus phases b - <a, s> of [B][dim+1] LWEs (key: s by default)."""
        key = self.s if key is None else key
        ph = (lwe[:, -1].astype(np.int64) - lwe_dot(lwe[:, :-1], key).astype(np.int64)) & MASK32
        return np.where(ph >= 1 << 31, ph - (1 << 32), ph)

    def decrypt(self, lwe: np.ndarray, key: np.ndarray | None = None) -> np.ndarray:
        """Messages round(phase / delta) mod 2t."""
        p = self.params
        ph = self.phases(lwe, key) & MASK32
        return ((ph + p.delta // 2) >> (32 - p.msg_bits - 1)) % (2 * p.t)


def test_vector(lut, params: TorusParams) -> np.ndarray:
    """Coefficient j carries lut[j // (N / t)] * delta (LUT_packing, cggi16.py:92-113)."""
    p = params
    lut = np.asarray(lut, dtype=np.int64)
    assert len(lut) == p.t
    return _u32(lut[np.arange(p.N) // (p.N // p.t)] * p.delta)


def generate_device_keys(params: TorusParams, rng: np.random.Generator, engine: Engine | None = None) -> "TorusKeys":
    """Torus keys whose random material is drawn on the GPU (vfhe_cuda_cggi_fft_gen_keys):
    the secret keys s and S come from `rng` on the host; the bootstrapping-key rows and
    the key-switching key are generated in HBM from the engine's ChaCha20 stream and
    stay there (bsk / ksk of the returned keys are None; bsk_d / ksk_d hold them)."""
    engine = engine or cuda_engine()
    ffi, lib = engine.ffi, engine.lib
    p = params
    s = rng.integers(0, 2, p.n).astype(np.int32)
    S = rng.integers(0, 2, p.N).astype(np.int32)
    bsk_d = torch.empty((p.n, 2 * p.bs_levels, 2, p.N), dtype=torch.int32, device="cuda")
    ksk_d = torch.empty((p.N, p.ks_levels, p.n + 1), dtype=torch.int32, device="cuda")
    ds, dS = torch.from_numpy(s).cuda(), torch.from_numpy(S).cuda()
    rc = lib.vfhe_cuda_cggi_fft_gen_keys(_p32(ffi, bsk_d), _p32(ffi, ksk_d), ffi.cast("int32_t*", ds.data_ptr()),
                                         ffi.cast("int32_t*", dS.data_ptr()), p.n, p.N, p.bs_base_log, p.bs_levels,
                                         p.ks_base_log, p.ks_levels, p.lwe_sigma, p.glwe_sigma,
                                         ffi.cast("void*", torch.cuda.current_stream().cuda_stream))
    if rc != 0:
        engine.check("cggi_fft_gen_keys")
        raise EngineError("cggi_fft_gen_keys")
    keys = TorusKeys(p, s, S, None, None)
    keys.bsk_d, keys.ksk_d = bsk_d, ksk_d
    return keys


def _p32(ffi, t: torch.Tensor):
    assert t.is_cuda and t.is_contiguous()
    return ffi.cast("uint32_t*", t.data_ptr())


class CggiFft:
    """Device-resident torus CGGI keys and the batched programmable bootstrap."""

    def __init__(self, keys: TorusKeys, engine: Engine | None = None):
        self.engine = engine or cuda_engine()
        self.ffi, self.lib = self.engine.ffi, self.engine.lib
        self.keys = keys
        p = self.params = keys.params
        bsk_d = getattr(keys, "bsk_d", None)
        if bsk_d is not None:  # generated on the device
            rows = bsk_d.reshape(-1, p.N)
        else:
            rows = torch.from_numpy(keys.bsk.reshape(-1, p.N).view(np.int32)).cuda()
        self.bsk_f = torch.empty((rows.shape[0], p.N // 2, 2), dtype=torch.float64, device="cuda")
        self._check(self.lib.vfhe_cuda_cggi_fft_to_fourier(self.ffi.cast("double*", self.bsk_f.data_ptr()),
                                                           _p32(self.ffi, rows), rows.shape[0], p.N, self._st()),
                    "cggi_fft_to_fourier")
        ksk_d = getattr(keys, "ksk_d", None)
        self.ksk = ksk_d if ksk_d is not None else torch.from_numpy(np.ascontiguousarray(keys.ksk).view(np.int32)).cuda()
        torch.cuda.synchronize()

    def _st(self, stream=None):
        return self.ffi.cast("void*", (stream or torch.cuda.current_stream()).cuda_stream)

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            self.engine.check(what)
            raise EngineError(what)

    def blind_rotate(self, lwe: torch.Tensor, tv: torch.Tensor, stream=None) -> torch.Tensor:
        """[B][n+1] LWEs under s -> [B][N+1] extracted LWEs under S (one persistent launch)."""
        p = self.params
        out = torch.empty((lwe.shape[0], p.N + 1), dtype=torch.int32, device="cuda")
        self._check(self.lib.vfhe_cuda_cggi_fft_bootstrap_batch(
            _p32(self.ffi, out), _p32(self.ffi, lwe), lwe.shape[0], self.ffi.cast("double*", self.bsk_f.data_ptr()),
            _p32(self.ffi, tv), p.n, p.N, p.bs_base_log, p.bs_levels, p.t, self._st(stream)), "cggi_fft_bootstrap")
        return out

    def keyswitch(self, ext: torch.Tensor, stream=None) -> torch.Tensor:
        p = self.params
        out = torch.empty((ext.shape[0], p.n + 1), dtype=torch.int32, device="cuda")
        self._check(self.lib.vfhe_cuda_cggi_fft_keyswitch_batch(
            _p32(self.ffi, out), _p32(self.ffi, ext), ext.shape[0], _p32(self.ffi, self.ksk), p.N, p.n,
            p.ks_base_log, p.ks_levels, self._st(stream)), "cggi_fft_keyswitch")
        return out

    def bootstrap(self, lwe: torch.Tensor, tv: torch.Tensor, stream=None) -> torch.Tensor:
        """Programmable bootstrap: blind rotation through tv, extraction, key switch."""
        return self.keyswitch(self.blind_rotate(lwe, tv, stream), stream)


def to_device(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def to_host(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)
