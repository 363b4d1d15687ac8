"""Uneven batched work list over the C ABI (vfhe_cuda_worklist_*).

Jobs of any mix of ring degree N and limb count L -- NTT -> product -> INTT chains and
GHS key switches -- are compiled once into device-resident row tables and run as three
persistent cooperative kernels per run (mode 0: forward transforms, products and
multiply-accumulates, inverse transforms and divisions, each walking the tables of
every transform pool with grid barriers between its phases), or as a CUDA graph of one
launch per stage per transform pool (mode 1, and the fallback for rows outside
2^8..2^16 points or split degrees above 4).  ``run_per_call`` executes the same jobs
one entry-point call each (vfhe_cuda_ntt_mul_intt_batch / vfhe_cuda_keyswitch_batch
with batch 1): the plain path the work list is measured against, and its parity
reference on the GPU.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from .arith import Ring
from .native import Engine, EngineError, cuda_engine


def _ptr(ffi, t: torch.Tensor):
    assert t.is_contiguous()
    return ffi.cast("uint64_t*", t.data_ptr())


@dataclass
class Job:
    """One work-list job.  chain: out = INTT(NTT(a) * NTT(b)), tensors [L][N];
    keyswitch: out = GHS key switch of ct [2][L][N] with ksk [L][2][L+1][N]."""

    kind: str
    ring: Ring
    L: int
    limbs: list[int]
    special: int | None
    out: torch.Tensor
    a: torch.Tensor
    b: torch.Tensor | None = None
    ksk: torch.Tensor | None = None
    _limbs_c: object = field(default=None, repr=False)

    @property
    def N(self) -> int:
        return self.ring.N

    def bytes_moved(self) -> int:
        """Algorithmic HBM bytes: inputs read once, outputs written once (keys read once)."""
        n, L = self.ring.N, self.L
        if self.kind == "chain":
            return 8 * n * L * 3
        return 8 * n * (2 * L + 2 * L + L * 2 * (L + 1))


class WorkList:
    """Compiled-once, replayed-many batch of independent jobs (one launch per run)."""

    def __init__(self, engine: Engine | None = None, mode: int = 0):
        self.engine = engine or cuda_engine()
        self.ffi, self.lib = self.engine.ffi, self.engine.lib
        self.handle = self.lib.vfhe_cuda_worklist_new()
        self.jobs: list[Job] = []
        self._check(self.lib.vfhe_cuda_worklist_set_mode(self.handle, mode), "worklist_set_mode")

    def _check(self, rc: int, what: str) -> None:
        if rc != 0:
            self.engine.check(what)
            raise EngineError(what)

    def add(self, job: Job) -> None:
        limbs = self.ffi.new("uint32_t[]", job.limbs)
        job._limbs_c = limbs
        if job.kind == "chain":
            rc = self.lib.vfhe_cuda_worklist_add_chain(self.handle, job.ring.NTT, _ptr(self.ffi, job.out),
                                                       _ptr(self.ffi, job.a), _ptr(self.ffi, job.b), limbs, job.L)
        else:
            rc = self.lib.vfhe_cuda_worklist_add_keyswitch(self.handle, job.ring.NTT, _ptr(self.ffi, job.out),
                                                           _ptr(self.ffi, job.a), limbs, job.L, job.special,
                                                           _ptr(self.ffi, job.ksk))
        self._check(rc, "worklist_add")
        self.jobs.append(job)

    def compile(self) -> None:
        self._check(self.lib.vfhe_cuda_worklist_compile(self.handle), "worklist_compile")

    def run(self, stream: torch.cuda.Stream | None = None) -> None:
        st = stream or torch.cuda.current_stream()
        self._check(self.lib.vfhe_cuda_worklist_run(self.handle, self.ffi.cast("void*", st.cuda_stream)),
                    "worklist_run")

    @property
    def launches(self) -> int:
        """Kernels one run launches (3 on the persistent path)."""
        return int(self.lib.vfhe_cuda_worklist_launches(self.handle))

    @property
    def persistent(self) -> bool:
        return bool(self.lib.vfhe_cuda_worklist_is_persistent(self.handle))

    @property
    def device_bytes(self) -> int:
        return int(self.lib.vfhe_cuda_worklist_device_bytes(self.handle))

    def close(self) -> None:
        if self.handle is not None:
            self.lib.vfhe_cuda_worklist_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def per_call_workspace(engine: Engine, jobs: list[Job]) -> torch.Tensor:
    need = max((engine.lib.vfhe_cuda_keyswitch_workspace_bytes(j.ring.NTT, 1, j.L) for j in jobs
                if j.kind == "keyswitch"), default=8)
    return torch.empty((need + 7) // 8, dtype=torch.int64, device="cuda")


def run_per_call(engine: Engine, jobs: list[Job], outs: list[torch.Tensor], ws: torch.Tensor,
                 stream: torch.cuda.Stream | None = None) -> int:
    """The same jobs through the one-job-per-call entry points; returns the call count."""
    ffi, lib = engine.ffi, engine.lib
    st = ffi.cast("void*", (stream or torch.cuda.current_stream()).cuda_stream)
    wsp = ffi.cast("void*", ws.data_ptr())
    for j, o in zip(jobs, outs):
        limbs = j._limbs_c if j._limbs_c is not None else ffi.new("uint32_t[]", j.limbs)
        if j.kind == "chain":
            rc = lib.vfhe_cuda_ntt_mul_intt_batch(j.ring.NTT, _ptr(ffi, o), _ptr(ffi, j.a), _ptr(ffi, j.b), 1,
                                                  limbs, j.L, st)
        else:
            rc = lib.vfhe_cuda_keyswitch_batch(j.ring.NTT, _ptr(ffi, o), _ptr(ffi, j.a), 1, limbs, j.L, j.special,
                                               _ptr(ffi, j.ksk), wsp, st)
        if rc != 0:
            engine.check("per-call job")
            raise EngineError("per-call job")
    return len(jobs)


def uneven_jobs(engine: Engine, count: int = 512, seed: int = 3, logn: tuple[int, int] = (12, 16),
                limbs: tuple[int, int] = (2, 24), device: str = "cuda") -> list[Job]:
    """The uneven workload: N uniform over 2^logn[0]..2^logn[1], L uniform over
    limbs[0]..limbs[1], half NTT->product->INTT chains and half key switches, every
    residue uniform in [0, q) from a seeded generator.  Primes: the 50-bit primes of
    Ring(N, prime_size=[50] * (L + 1)) at the ring's default split degree (the key
    switch's special prime is the (L+1)-th)."""
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    rings: dict[int, Ring] = {}
    jobs = []
    for _ in range(count):
        n = 1 << int(rng.integers(logn[0], logn[1] + 1))
        L = int(rng.integers(limbs[0], limbs[1] + 1))
        kind = "chain" if rng.random() < 0.5 else "keyswitch"
        if n not in rings:
            rings[n] = Ring(n, prime_size=[50] * (limbs[1] + 1), engine=engine)
        R = rings[n]
        idx = list(R.prime_indices[:L])
        qs = R.primes[: L + 1]

        def uniform(shape, prime_axis, nprimes):
            t = torch.empty(shape, dtype=torch.int64, device=device)
            for k in range(nprimes):
                sl = [slice(None)] * len(shape)
                sl[prime_axis] = k
                t[tuple(sl)].random_(0, qs[k], generator=gen)
            return t

        if kind == "chain":
            a = uniform((L, n), 0, L)
            b = uniform((L, n), 0, L)
            jobs.append(Job("chain", R, L, idx, None, torch.empty_like(a), a, b=b))
        else:
            ct = uniform((2, L, n), 1, L)
            ksk = uniform((L, 2, L + 1, n), 2, L + 1)
            jobs.append(Job("keyswitch", R, L, idx, R.prime_indices[L], torch.empty_like(ct), ct, ksk=ksk))
    return jobs


def run_job_on_engine(engine: Engine, job: Job) -> np.ndarray:
    """One job recomputed through the one-op-per-call cdef surface of `engine` (any
    engine: the cuda engine, or a CPU library exporting the same cdef), as the
    reference's callers would run it:
    chain     = polynomial_RNSc_to_RNS of both operands, polynomial_mul_RNS_polynomial,
                polynomial_RNS_to_RNSc (rns_polynomial.c:311-356, 582-614);
    keyswitch = mlwe_RNSc_GHS_hybrid_keyswitch of the rank-1 sample with one key
                (mlwe.c:557-598).
    Inputs are read from the job's tensors; returns the output rows."""
    from .arith import Polynomial
    from .arith import repr as prepr
    from .mlwe import MLWE, MLWE_Scheme, MLWE_Set

    def host(t):
        return t.cpu().numpy().view(np.uint64)

    def poly(R, rows):
        p = Polynomial(R)
        p.set_rows(rows)
        p.rns_mask = R.mask
        p.repr = prepr.coeff
        return p

    L = job.L
    if job.kind == "chain":
        R = Ring(job.N, prime_size=[50] * L, primes=job.ring.primes[:L], split_degree=job.ring.split_degree,
                 engine=engine)
        c = poly(R, host(job.a)) * poly(R, host(job.b))
        c.to_coeff()
        return c.rows()
    R = Ring(job.N, prime_size=[50] * (L + 1), primes=job.ring.primes[: L + 1], split_degree=job.ring.split_degree,
             engine=engine)
    s = MLWE_Scheme(R, special_primes=1, module_rank=1, max_lvl=1)
    ct, ksk = host(job.a), host(job.ksk)
    c = MLWE(s)
    c.set_component_rows(0, ct[0])
    c.set_component_rows(1, ct[1])
    c.repr = prepr.coeff
    comps = []
    for j in range(L):
        k = MLWE(s, ring=s.special_rings[0])
        k.set_component_rows(0, ksk[j][0])
        k.set_component_rows(1, ksk[j][1])
        k.repr = prepr.ntt
        comps.append(k)
    out = s.keyswitch(c, MLWE_Set([comps]))
    return np.stack([out.component_rows(0), out.component_rows(1)])
