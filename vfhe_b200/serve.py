"""Serving loop over the C ABI (vfhe_cuda_server_*): continuous batching of mixed CKKS
and CGGI requests with device-resident keys and ciphertexts and an HBM budget.

The loop itself is native (csrc/server.cu: one worker thread, per-class queues,
stream slots, stream-ordered scratch, completion events).  This module registers
parameter classes, submits requests and collects latencies; ``poisson_arrivals`` and
``ServingMix`` build the synthetic request streams the benchmark sweeps.  The plain
one-call-per-request path is the same server with ``max_batch=1`` and one stream.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .native import Engine, EngineError, cuda_engine


def _p(ffi, t: torch.Tensor | None):
    if t is None:
        return ffi.NULL
    assert t.is_cuda and t.is_contiguous()
    return ffi.cast("uint64_t*", t.data_ptr())


class Server:
    def __init__(self, budget_bytes: int, streams: int = 4, max_batch: int = 64, engine: Engine | None = None):
        self.engine = engine or cuda_engine()
        self.ffi, self.lib = self.engine.ffi, self.engine.lib
        self.handle = self.lib.vfhe_cuda_server_new(int(budget_bytes), streams, max_batch)
        if self.handle == self.ffi.NULL:
            self.engine.check("server_new")
            raise EngineError("server_new")
        self._keep: list = []

    def reserve(self, nbytes: int) -> None:
        if self.lib.vfhe_cuda_server_reserve(self.handle, int(nbytes)) != 0:
            self.engine.check("server_reserve")
            raise EngineError("server_reserve")

    def note_resident(self, nbytes: int) -> None:
        self.lib.vfhe_cuda_server_note_resident(self.handle, int(nbytes))

    def ckks_class(self, ring, special: int, rlk: torch.Tensor | None) -> int:
        limbs = self.ffi.new("uint32_t[]", list(ring.prime_indices))
        c = self.lib.vfhe_cuda_server_ckks_class(self.handle, ring.NTT, limbs, ring.ell, special, _p(self.ffi, rlk))
        if c < 0:
            self.engine.check("server_ckks_class")
            raise EngineError("server_ckks_class")
        self._keep.append(rlk)
        return c

    def cggi_class(self, ring, special: int, n: int, bk: torch.Tensor, tv: torch.Tensor, torus_base: int,
                   max_count: int) -> int:
        limbs = self.ffi.new("uint32_t[]", list(ring.prime_indices))
        c = self.lib.vfhe_cuda_server_cggi_class(self.handle, ring.NTT, limbs, ring.ell, special, n, _p(self.ffi, bk),
                                                 _p(self.ffi, tv), torus_base, max_count)
        if c < 0:
            self.engine.check("server_cggi_class")
            raise EngineError("server_cggi_class")
        self._keep += [bk, tv]
        return c

    def torus_class(self, dev, tv: torch.Tensor, max_count: int) -> int:
        """A torus CGGI class over the device keys of a CggiFft (programmable bootstrap
        through the test vector tv, key switch back to the LWE key)."""
        p = dev.params
        c = self.lib.vfhe_cuda_server_torus_class(
            self.handle, self.ffi.cast("double*", dev.bsk_f.data_ptr()), self.ffi.cast("uint32_t*", tv.data_ptr()),
            self.ffi.cast("uint32_t*", dev.ksk.data_ptr()), p.n, p.N, p.bs_base_log, p.bs_levels, p.ks_base_log,
            p.ks_levels, p.t, max_count)
        if c < 0:
            self.engine.check("server_torus_class")
            raise EngineError("server_torus_class")
        self._keep += [dev, tv]
        return c

    def submit_torus(self, cls: int, out: torch.Tensor, lwe: torch.Tensor) -> int:
        return self._ok(self.lib.vfhe_cuda_server_submit_torus(self.handle, cls, self.ffi.cast("uint32_t*", out.data_ptr()),
                                                               self.ffi.cast("uint32_t*", lwe.data_ptr()),
                                                               lwe.shape[0]))

    def submit_mul(self, cls: int, out: torch.Tensor, ct1: torch.Tensor, ct2: torch.Tensor) -> int:
        return self._ok(self.lib.vfhe_cuda_server_submit_ckks_mul(self.handle, cls, _p(self.ffi, out),
                                                                  _p(self.ffi, ct1), _p(self.ffi, ct2)))

    def submit_rotate(self, cls: int, out: torch.Tensor, ct: torch.Tensor, gen: int, gk: torch.Tensor) -> int:
        return self._ok(self.lib.vfhe_cuda_server_submit_ckks_rotate(self.handle, cls, _p(self.ffi, out),
                                                                     _p(self.ffi, ct), gen, _p(self.ffi, gk)))

    def submit_cggi(self, cls: int, out_a: torch.Tensor, out_b: torch.Tensor, a: torch.Tensor, b: torch.Tensor) -> int:
        return self._ok(self.lib.vfhe_cuda_server_submit_cggi(self.handle, cls, _p(self.ffi, out_a),
                                                              _p(self.ffi, out_b), _p(self.ffi, a), _p(self.ffi, b),
                                                              a.shape[0]))

    def _ok(self, rid: int) -> int:
        if rid < 0:
            raise EngineError("server submit rejected (bad class or arguments)")
        return int(rid)

    def wait(self, rid: int, timeout_ms: float | None = None) -> float:
        """Latency (ms) of request `rid` once it finished.  Raises EngineError when it
        failed or was cancelled, TimeoutError when `timeout_ms` ran out (the request is
        kept: wait again or cancel it)."""
        ms = self.ffi.new("double*")
        rc = self.lib.vfhe_cuda_server_wait_for(self.handle, rid, -1.0 if timeout_ms is None else float(timeout_ms), ms)
        if rc == 2:
            raise TimeoutError(f"server request {rid} not finished after {timeout_ms} ms")
        if rc == 3:
            raise EngineError(f"server request {rid} was cancelled")
        if rc != 0:
            self.engine.check("server request")
            raise EngineError(f"server request {rid} failed")
        return float(ms[0])

    def poll(self, rid: int, timeout_ms: float = 0.0) -> int:
        """Raw wait status: 0 done, 1 failed or unknown, 2 not finished yet, 3 cancelled
        (a finished request is forgotten, as with wait)."""
        return int(self.lib.vfhe_cuda_server_wait_for(self.handle, rid, float(timeout_ms), self.ffi.NULL))

    def cancel(self, rid: int) -> bool:
        """Cancel a request no batch has taken yet; False when it already runs or finished."""
        rc = self.lib.vfhe_cuda_server_cancel(self.handle, rid)
        if rc < 0:
            raise EngineError(f"unknown server request {rid}")
        return rc == 0

    def pause(self, paused: bool = True) -> None:
        """Hold (or resume) the admission of queued requests into batches."""
        self.lib.vfhe_cuda_server_pause(self.handle, 1 if paused else 0)

    def set_batch_timeout(self, ms: float) -> None:
        """Fail the requests of any batch still running `ms` after its launch (0: never)."""
        if self.lib.vfhe_cuda_server_set_batch_timeout(self.handle, float(ms)) != 0:
            raise EngineError("bad batch timeout")

    def inject_fault(self, kind: str, count: int = 1) -> None:
        """Host-side fault injection for tests: 'launch' (the next batch launches fail),
        'alloc' (the next scratch allocations fail; batches are re-queued) or 'stall'
        (the next batches' completions go unobserved until the batch deadline)."""
        k = {"launch": 1, "alloc": 2, "stall": 3}[kind]
        if self.lib.vfhe_cuda_server_inject_fault(self.handle, k, count) != 0:
            raise EngineError("fault injection refused")

    def fault_stats(self) -> dict:
        out = self.ffi.new("uint64_t[4]")
        self.lib.vfhe_cuda_server_fault_stats(self.handle, out)
        return {"expired_batches": out[0], "alloc_retries": out[1], "cancelled": out[2], "injected_pending": out[3]}

    def stats(self) -> dict:
        out = self.ffi.new("uint64_t[5]")
        self.lib.vfhe_cuda_server_stats(self.handle, out)
        return {"completed": out[0], "failed": out[1], "batches": out[2], "batched_requests": out[3],
                "hbm_bytes_in_use": out[4]}

    def close(self) -> None:
        if self.handle is not None:
            self.lib.vfhe_cuda_server_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_arrivals(rate: float, count: int, rng: np.random.Generator) -> np.ndarray:
    """Arrival times (s, from 0) of a Poisson stream; rate <= 0 means all at t = 0."""
    if rate <= 0:
        return np.zeros(count)
    return np.cumsum(rng.exponential(1.0 / rate, count))


def _uniform(shape, qs, axis, gen, device="cuda"):
    t = torch.empty(shape, dtype=torch.int64, device=device)
    for k, q in enumerate(qs):
        sl = [slice(None)] * len(shape)
        sl[axis] = k
        t[tuple(sl)].random_(0, q, generator=gen)
    return t


@dataclass
class CkksParams:
    N: int
    L: int
    mul_cls: int = -1
    rot_cls: int = -1
    ring: object = None
    rlk: torch.Tensor | None = None
    gks: dict = field(default_factory=dict)
    cts: list = field(default_factory=list)   # NTT-domain inputs of the multiply [2][L][N]
    rcts: list = field(default_factory=list)  # coefficient-domain inputs of the rotation [2][L-1][N]


@dataclass
class CggiParams:
    N: int
    n: int
    cls: int = -1
    a: torch.Tensor | None = None
    b: torch.Tensor | None = None


class ServingMix:
    """Synthetic serving setup: CKKS parameter classes (N, L) with a relinearisation key,
    Galois keys and a pool of input ciphertexts each (every residue uniform from a seeded
    generator: throughput and latency do not depend on key values), and one CGGI class
    with a pool of LWE inputs.  cggi_kind "torus" (the CGGI16 parameter set: n, N,
    gadget 2^7 x 3, key switch 2^2 x 8) uses real keys and encryptions of random 4-bit
    messages; "rns" uses the RNS-gadget CGGI16 with uniform key material."""

    def __init__(self, engine: Engine, ckks=((2**13, 4), (2**14, 9), (2**15, 16), (2**16, 24)),
                 cggi=(1024, 630), cggi_max=1024, pool: int = 4, gens: int = 2, seed: int = 7, with_cggi=True,
                 cggi_kind: str = "torus"):
        from .arith import Ring

        self.engine = engine
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed)
        self.rng = np.random.default_rng(seed)
        self.ckks: list[CkksParams] = []
        self.resident = 0
        for N, L in ckks:
            # ciphertext primes: one 50-bit base prime and L - 1 primes of 40 bits; one
            # 50-bit special prime (the CKKS chain of the benchmark, other N and L)
            sizes = [50] + [40] * (L - 1)
            R = Ring(N, prime_size=sizes + [50], split_degree=1, engine=engine)
            q = R.primes
            ring_L = Ring(N, primes=q[:L], prime_size=sizes, split_degree=1, engine=engine)
            ring_R = Ring(N, primes=q[: L - 1], prime_size=sizes[:-1], split_degree=1, engine=engine)
            p = CkksParams(N, L, ring=(R, ring_L, ring_R))
            ext = q[:L] + [q[L]]
            p.rlk = _uniform((L, 2, L + 1, N), ext, 2, gen)
            ext_r = q[: L - 1] + [q[L]]
            for g in range(gens):
                p.gks[5 ** (g + 1) % (2 * N)] = _uniform((L - 1, 2, L, N), ext_r, 2, gen)
            p.cts = [_uniform((2, L, N), q[:L], 1, gen) for _ in range(pool)]
            p.rcts = [_uniform((2, L - 1, N), q[: L - 1], 1, gen) for _ in range(pool)]
            self.resident += 8 * (p.rlk.numel() + sum(k.numel() for k in p.gks.values()) +
                                  sum(c.numel() for c in p.cts + p.rcts))
            p.special = R.prime_indices[L]
            self.ckks.append(p)
        self.cggi = None
        self.cggi_kind = cggi_kind
        if with_cggi and cggi_kind == "torus":
            from .cggi_fft import CggiFft, TorusKeys, TorusParams, test_vector
            from .cggi_fft import to_device as to_device32

            N, n = cggi
            tp = TorusParams(n=n, N=N)
            keys = TorusKeys.generate(tp, self.rng)
            cg = CggiParams(N, n)
            cg.dev = CggiFft(keys, engine)
            cg.lut = self.rng.integers(0, tp.t, tp.t)
            cg.tv = to_device32(test_vector(cg.lut, tp))
            cg.msgs = self.rng.integers(0, tp.t, cggi_max)
            cg.lwe = to_device32(keys.encrypt(cg.msgs, self.rng))
            cg.keys = keys
            cg.max = cggi_max
            self.resident += cg.dev.bsk_f.numel() * 8 + cg.dev.ksk.numel() * 4 + cg.lwe.numel() * 4
            self.cggi = cg
        elif with_cggi:
            N, n = cggi
            Rc = Ring(N, prime_size=[50, 50, 50], split_degree=1, engine=engine)
            q = Rc.primes
            cg = CggiParams(N, n)
            cg.ring = Ring(N, primes=q[:2], prime_size=[50, 50], split_degree=1, engine=engine)
            cg.special = Rc.prime_indices[2]
            cg.bk = _uniform((n, 4, 2, 3, N), q, 3, gen)
            cg.tv = _uniform((2, 2, N), q[:2], 1, gen)
            cg.a = _uniform((cggi_max, 2, n), q[:2], 1, gen)
            cg.b = _uniform((cggi_max, 2), q[:2], 1, gen)
            cg.max = cggi_max
            self.resident += 8 * (cg.bk.numel() + cg.tv.numel() + cg.a.numel() + cg.b.numel())
            self.cggi = cg

    def register(self, server: Server) -> None:
        server.note_resident(self.resident)
        for p in self.ckks:
            _, ring_L, ring_R = p.ring
            p.mul_cls = server.ckks_class(ring_L, p.special, p.rlk)
            p.rot_cls = server.ckks_class(ring_R, p.special, None)
        if self.cggi is not None and self.cggi_kind == "torus":
            cg = self.cggi
            cg.cls = server.torus_class(cg.dev, cg.tv, cg.max)
        elif self.cggi is not None:
            cg = self.cggi
            cg.cls = server.cggi_class(cg.ring, cg.special, cg.n, cg.bk, cg.tv, 16, cg.max)

    def requests(self, count: int, seed: int, ckks_share: float = 0.8, cggi_counts=(1, 1024)):
        """A reproducible list of (kind, class-param index, input index, extra) requests."""
        rng = np.random.default_rng(seed)
        out = []
        for _ in range(count):
            if self.cggi is None or rng.random() < ckks_share:
                pi = int(rng.integers(len(self.ckks)))
                p = self.ckks[pi]
                if rng.random() < 0.5:
                    out.append(("mul", pi, int(rng.integers(len(p.cts))), int(rng.integers(len(p.cts)))))
                else:
                    gens = sorted(p.gks)
                    out.append(("rot", pi, int(rng.integers(len(p.rcts))), gens[int(rng.integers(len(gens)))]))
            else:
                lo, hi = np.log2(cggi_counts[0]), np.log2(cggi_counts[1])
                c = int(round(2 ** rng.uniform(lo, hi)))
                out.append(("cggi", -1, c, int(rng.integers(0, self.cggi.max - c + 1))))
        return out

    def output_for(self, req) -> tuple:
        kind, pi, x, y = req
        if kind == "mul":
            p = self.ckks[pi]
            return (torch.empty((2, p.L - 1, p.N), dtype=torch.int64, device="cuda"),)
        if kind == "rot":
            p = self.ckks[pi]
            return (torch.empty((2, p.L - 1, p.N), dtype=torch.int64, device="cuda"),)
        cg = self.cggi
        if self.cggi_kind == "torus":
            return (torch.empty((x, cg.n + 1), dtype=torch.int32, device="cuda"),)
        return (torch.empty((x, 2, cg.N), dtype=torch.int64, device="cuda"),
                torch.empty((x, 2), dtype=torch.int64, device="cuda"))

    def submit(self, server: Server, req, outs) -> int:
        kind, pi, x, y = req
        if kind == "mul":
            p = self.ckks[pi]
            return server.submit_mul(p.mul_cls, outs[0], p.cts[x], p.cts[y])
        if kind == "rot":
            p = self.ckks[pi]
            return server.submit_rotate(p.rot_cls, outs[0], p.rcts[x], y, p.gks[y])
        cg = self.cggi
        if self.cggi_kind == "torus":
            return server.submit_torus(cg.cls, outs[0], cg.lwe[y:y + x])
        return server.submit_cggi(cg.cls, outs[0], outs[1], cg.a[y:y + x], cg.b[y:y + x])


def run_stream(mix: ServingMix, server: Server, reqs, arrivals: np.ndarray, keep_outputs: bool = False) -> dict:
    """Submit `reqs` at `arrivals` (seconds from start), wait for all, report latencies."""
    outs = [mix.output_for(r) for r in reqs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ids = []
    for r, o, ta in zip(reqs, outs, arrivals):
        while time.perf_counter() - t0 < ta:
            pass
        ids.append(mix.submit(server, r, o))
    lat = np.array([server.wait(i) for i in ids])
    wall = time.perf_counter() - t0
    res = {"requests": len(reqs), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "mean_ms": float(lat.mean()), "throughput_rps": len(reqs) / wall, "wall_s": wall}
    if keep_outputs:
        res["outputs"] = outs
    return res
