"""Benchmark: batched CKKS multiply -> relinearise -> rescale -> rotate on B200.

Workload (one "step"): 256 ciphertext pairs in Z_Q[X]/(X^16384 + 1), one 50-bit base
prime + eight 40-bit primes (L = 9) plus one 50-bit special prime, scale 2^40,
ternary secret, sigma 3.2 errors, 2^13 slots uniform in the unit disk.  Each pair is
multiplied, relinearised, rescaled to L = 8 and rotated by a step drawn from
{1, 2, 4, ..., 2^12} (13 Galois keys resident in HBM).  All inputs are synthetic
from fixed seeds.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

Prints one JSON line (rank 0).  ``value`` is pairs per second over all ranks with
ciphertexts already in HBM; ``e2e`` adds the host->device copy of each step's input
ciphertexts (uint64 residue rows) from pinned memory and the device->host copy of its
results; the same step moving ciphertexts in the compact wire format (residues at their
primes' bit lengths, as a sender would ship them) is timed beside it.  The
reference arm runs the reference's own CPU library (built from its sources into
oracle/_ref/) on the same workload, one process per host core.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
N_DEG = 2**14
PRIME_SIZES = [50] + [40] * 8 + [50]
PAIRS = 256
NTT16_POLYS = 64  # polynomials per N = 2^16, L = 24 transform launch
# DRAM bytes (read + write) of one digit-transform launch, per (schedule, rows), from an
# ncu capture of that launch (dram__bytes_read.sum + dram__bytes_write.sum over its kernels)
MEASURED_TRAFFIC = {("k_col_f<4,0> + k_tile_fwd_f<10,1>", 2560): 1230588672}
STEPS_SET = [1 << i for i in range(13)]
SCALE = 2.0**40
SEED = 20261203
CONFIG = {
    "workload": "CKKS mul+relin+rescale+rotate, N=2^14, L=9 (1x50-bit + 8x40-bit) + 1 special 50-bit prime, "
                "scale 2^40, 256 ciphertext pairs per step, rotation steps 2^0..2^12",
    "N": N_DEG,
    "L": 9,
    "special_primes": 1,
    "pairs_per_step": PAIRS,
    "l2_policy": "inputs larger than L2 (1.2 GB of ciphertexts per step)",
    "parallelism": "replicas, ciphertext pairs sharded by rank (no data-path collective): one job of "
                   "world x 256 pairs from one seed, rank r takes pairs [256 r, 256 (r + 1))",
}


# ----------------------------------------------------------------------------- setup
def pair_share(rank: int, pairs_per_rank: int) -> range:
    """Global indices of the ciphertext pairs one rank processes.  The job is
    world x pairs_per_rank pairs drawn from one seed; rank r takes the r-th block of
    pairs_per_rank, so the shares are disjoint and together are the whole job (weak
    scaling: the per-rank share is fixed as ranks are added)."""
    return range(rank * pairs_per_rank, (rank + 1) * pairs_per_rank)


def build_workload(engine, pairs: int, seed: int, first_pair: int = 0, gk_steps=STEPS_SET, n: int = N_DEG,
                   prime_sizes=PRIME_SIZES):
    """Keys and ciphertexts through the reference API mirror (seeded, engine-independent).

    The keys come from `seed` alone, so every rank holds the same ones; pair p of the job
    (its two ciphertexts and its rotation step) comes from the seed sequence (seed, p),
    so a pair is the same whichever rank draws it.  Returns pairs first_pair ..
    first_pair + pairs - 1."""
    from vfhe_b200.arith import Ring
    from vfhe_b200.fhe import CKKS_Scheme
    from vfhe_b200.native import use_engine

    with use_engine(engine):
        rng = np.random.default_rng(seed)
        R = Ring(n, prime_size=prime_sizes, split_degree=1)
        s = CKKS_Scheme(R, scaling_factor=SCALE, special_primes=1)
        key = s.key_gen_uniform_ternary(3.2, rng)
        rlk = s.gen_rlk(key, key, lvl=0, rng=rng)
        gks = {k: s.gen_ksk_automorphism(key, key, s.galois_gen(k), lvl=1, rng=rng) for k in gk_steps}
        steps, zs, cts = [], [], []
        for p in range(first_pair, first_pair + pairs):
            prng = np.random.default_rng([seed, p])
            steps.append(int(prng.choice(gk_steps)))
            for _ in range(2):
                z = np.sqrt(prng.random(n // 2)) * np.exp(2j * np.pi * prng.random(n // 2))
                zs.append(z)
                cts.append(s.encrypt(s.encode(list(z)), key, rng=prng))
        return s, key, rlk, gks, steps, zs, cts


def decoded_error(s, key, ct, expect, delta) -> float:
    dec = np.array(s.decode(s.decrypt(ct, key), scaling_factor=delta))
    return float(np.max(np.abs(dec - expect)))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms over the with-block.

    Entering waits (at most 10 s) for the sampler's first line, so sampling is running
    when the timed region starts; leaving waits (at most 1 s) for one more line, so a
    region shorter than the sampling period still gets a sample taken at its end.  Only
    lines that arrive after the first one are kept."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 50

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.kept: list[str] = []
        self.thread = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line)

    def _wait_lines(self, n: int, limit_s: float) -> None:
        t0 = time.monotonic()
        while len(self.lines) < n and time.monotonic() - t0 < limit_s and self.thread.is_alive():
            time.sleep(0.005)

    def __enter__(self):
        import threading

        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.PERIOD_MS)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return self
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        self._wait_lines(1, 10.0)
        self.first = len(self.lines)
        return self

    def __exit__(self, *exc):
        if self.proc is None:
            return
        self._wait_lines(self.first + 1, 1.0)
        self.kept = list(self.lines[self.first:])
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)

    def summary(self) -> dict:
        if not self.kept:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.kept:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ----------------------------------------------------------------------------- cpu legs
def _ref_library() -> tuple[Path, str]:
    ifma = "avx512ifma" in Path("/proc/cpuinfo").read_text()
    name = "avx512ifma" if ifma else "portable"
    return ROOT / "oracle" / "_ref" / f"libvfhe_ref_{name}.so", name


def _cpu_library() -> tuple[Path, str, str]:
    """(library, engine name, kind) of the CPU implementation that the reference arm and
    the one-core baseline time: the reference's own library compiled from its sources
    (oracle/_ref, kind "reference"), else the oracle's C restatement of the same path
    (kind "port"), compiled here if needed."""
    lib, name = _ref_library()
    if lib.exists():
        return lib, name, "reference"
    port = ROOT / "oracle" / "_build" / "libvfhe_oracle.so"
    src = ROOT / "oracle" / "vfhe_oracle.c"
    if not port.exists() or port.stat().st_mtime < src.stat().st_mtime:
        port.parent.mkdir(exist_ok=True)
        subprocess.run(["gcc", "-O2", "-std=gnu11", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(port),
                        str(src), "-lm"], check=True)
    return port, "oracle", "port"


def _ref_worker(args) -> dict:
    """One host core: the CPU implementation (_cpu_library), a bounded number of pairs,
    warmup + timed steps."""
    pairs, warmup, steps, seed, time_budget = args
    from vfhe_b200.native import Engine

    lib, name, kind = _cpu_library()
    eng = Engine(lib, name if kind == "port" else None)
    s, key, rlk, gks, rot, zs, cts = build_workload(eng, pairs, seed, gk_steps=sorted(set(STEPS_SET[:2])))

    def one_step():
        for p in range(pairs):
            prod = s.multiply(cts[2 * p], cts[2 * p + 1], rlk)
            prod.round_division(lvl=1)
            k = STEPS_SET[p % 2]
            s.automorphism(prod, s.galois_gen(k), gks[k])

    for _ in range(warmup):
        one_step()
    t0 = time.perf_counter()
    done = 0
    for _ in range(steps):
        one_step()
        done += 1
        if time_budget and time.perf_counter() - t0 > time_budget:
            break
    return {"elapsed": time.perf_counter() - t0, "pairs": pairs * done, "engine": name}


def _ref_poly(R, rows):
    from vfhe_b200.arith import Polynomial
    from vfhe_b200.arith import repr as prepr

    p = Polynomial(R)
    p.set_rows(rows)
    p.rns_mask = R.mask
    p.repr = prepr.coeff
    return p


def _cpu_ntt_worker(args) -> dict:
    """One host core: the reference library's forward transform of every limb of one
    polynomial (polynomial_RNSc_to_RNS, rns_polynomial.c:582-614) at N = 2^logn with
    `limbs` 50-bit primes, repeated for `seconds` after one warm-up call."""
    logn, limbs, split, seconds, seed = args
    from vfhe_b200.arith import Polynomial, Ring
    from vfhe_b200.native import Engine

    lib, name = _ref_library()
    eng = Engine(lib)
    R = Ring(2**logn, prime_size=[50] * limbs, split_degree=split, engine=eng)
    rng = np.random.default_rng(seed)
    src = _ref_poly(R, np.stack([rng.integers(0, q, R.N, dtype=np.uint64) for q in R.primes]))
    out = Polynomial(R)
    eng.lib.polynomial_RNSc_to_RNS(out.obj, src.obj)
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        eng.lib.polynomial_RNSc_to_RNS(out.obj, src.obj)
        done += 1
    return {"units": done * limbs, "elapsed": time.perf_counter() - t0, "engine": name}


def _cpu_roundtrip_worker(args) -> dict:
    """One host core: the reference library's NTT -> incomplete product -> INTT chain of
    one pair at N = 4096, L = 3 (polynomial_RNSc_to_RNS x 2, polynomial_mul_RNS_polynomial,
    polynomial_RNS_to_RNSc), repeated for `seconds`."""
    split, seconds, seed = args
    from vfhe_b200.arith import Polynomial, Ring
    from vfhe_b200.native import Engine

    lib, name = _ref_library()
    eng = Engine(lib)
    R = Ring(4096, prime_size=[50] * 3, split_degree=split, engine=eng)
    rng = np.random.default_rng(seed)
    a, b = (_ref_poly(R, np.stack([rng.integers(0, q, R.N, dtype=np.uint64) for q in R.primes])) for _ in range(2))
    P = [Polynomial(R) for _ in range(3)]
    rl = eng.lib
    done, t0 = -1, time.perf_counter()
    while done < 0 or time.perf_counter() - t0 < seconds:
        if done == 0:
            t0 = time.perf_counter()  # the first chain is the warm-up
        rl.polynomial_RNSc_to_RNS(P[0].obj, a.obj)
        rl.polynomial_RNSc_to_RNS(P[1].obj, b.obj)
        rl.polynomial_mul_RNS_polynomial(P[2].obj, P[0].obj, P[1].obj)
        rl.polynomial_RNS_to_RNSc(P[2].obj, P[2].obj)
        done += 1
    return {"units": done, "elapsed": time.perf_counter() - t0, "engine": name}


class CpuPool:
    """Spawned processes, one per host core, for the reference's all-cores figures
    (spawned, not forked: the parent holds a CUDA context)."""

    def __init__(self):
        self.cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        self.pool = None

    def rate(self, worker, args: tuple, seed: int) -> dict:
        """units/s over all cores: every process runs `worker` for the same time budget."""
        import multiprocessing as mp

        if self.pool is None:
            self.pool = mp.get_context("spawn").Pool(self.cores)
        res = self.pool.map(worker, [args + (seed + w,) for w in range(self.cores)])
        return {"value": sum(r["units"] for r in res) / max(r["elapsed"] for r in res), "cores": self.cores,
                "engine": res[0]["engine"]}

    def close(self):
        if self.pool is not None:
            self.pool.close()
            self.pool.join()
            self.pool = None


def cpu_baseline(time_budget: float = 15.0) -> dict:
    """The CPU implementation (_cpu_library), one core, bounded sample of the same
    workload (pairs/s)."""
    lib, name, kind = _cpu_library()
    r = _ref_worker((1, 1, 100000, SEED + 7, time_budget))
    what = f"the reference's {name} engine" if kind == "reference" else "the oracle port"
    return {"value": r["pairs"] / r["elapsed"], "unit": "pairs/s", "cores": 1, "kind": kind,
            "sample": f"{r['pairs']} pairs of the same workload on {what}, one thread, {r['elapsed']:.1f} s"}


def run_reference_arm(args) -> None:
    import multiprocessing as mp

    lib, name, kind = _cpu_library()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    workers = max(1, min(cores, 96))
    ctx = mp.get_context("spawn")
    steps = args.steps
    with ctx.Pool(workers) as pool:
        res = pool.map(_ref_worker, [(1, args.warmup, steps, SEED + 1000 + w, 0) for w in range(workers)])
    elapsed = max(r["elapsed"] for r in res)
    total = sum(r["pairs"] for r in res)
    value = total / elapsed
    line = {
        "impl": "reference", "metric": "CKKS mul+relin+rescale/s", "value": value, "unit": "pairs/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (RNS residues < 2^50)",
        "data": "synthetic (seeded)", "config": dict(CONFIG, pairs_per_step=workers),
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": workers, "kind": kind,
                         "sample": f"{workers} processes x 1 pair per step on "
                                   + (f"the reference's {name} engine" if kind == "reference" else "the oracle port")},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------------------------- profiling
PROFILE_LEG = "ckks"


def profile_range(args, leg: str, start: bool) -> None:
    """Open/close the profiler's capture range (ncu --profile-from-start off) around the
    timed region of the leg chosen with --profile-leg."""
    if PROFILE_LEG != leg:
        return
    import torch

    torch.cuda.synchronize()
    if start:
        torch.cuda.profiler.start()
    else:
        torch.cuda.profiler.stop()


# ----------------------------------------------------------------------------- ranks
def max_over_ranks(ms: float, dist, device) -> float:
    """The slowest rank's time: every rank enters this reduction in the same order."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, ms: float) -> float:
    """Units per second over all ranks (weak scaling: every rank does units_per_rank)."""
    return world * units_per_rank / (ms * 1e-3)


# ----------------------------------------------------------------------------- gpu arm
def worklist_leg(eng, count: int, reps: int, cpu_budget: float = 0.0) -> dict:
    """Uneven batch: `count` jobs, N in 2^12..2^16, L in 2..24, half NTT->product->INTT
    chains and half key switches, as one persistent work-list launch per run, beside
    the graph of per-pool launches and one call per job."""
    import torch

    from vfhe_b200.worklist import WorkList, per_call_workspace, run_per_call, uneven_jobs

    jobs = uneven_jobs(eng, count=count, seed=SEED + 3)
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(mode, profile):
        w = WorkList(eng, mode=mode)
        for j in jobs:
            w.add(j)
        w.run(stream)  # compile (+ capture) + first run
        torch.cuda.synchronize()
        if profile:
            profile_range(None, PROFILE_LEG, True)
        ev0.record(stream)
        for _ in range(reps):
            w.run(stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        if profile:
            profile_range(None, PROFILE_LEG, False)
        return w, ev0.elapsed_time(ev1) / reps

    wg, ms_graph = timed(1, PROFILE_LEG == "worklist_graph")
    graph_launches = wg.launches
    graph_out = [j.out.clone() for j in jobs]
    wg.close()
    wl, ms_wl = timed(0, PROFILE_LEG == "worklist")
    ph = eng.ffi.new("double[6]")
    phases = None
    if eng.lib.vfhe_cuda_worklist_phase_ms(wl.handle, ph) == 0:
        phases = dict(zip(["forward_columns_and_one_pass", "forward_tiles_two_pass", "products_and_macs",
                           "inverse_tiles", "inverse_columns_and_one_pass_divisions", "divisions_two_pass"],
                          [round(ph[k], 3) for k in range(6)]))
    persistent_exact = all(torch.equal(j.out, g) for j, g in zip(jobs, graph_out))
    del graph_out
    outs = [torch.empty_like(j.out) for j in jobs]
    ws = per_call_workspace(eng, jobs)
    calls = run_per_call(eng, jobs, outs, ws, stream)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(reps):
        run_per_call(eng, jobs, outs, ws, stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms_pc = ev0.elapsed_time(ev1) / reps
    exact = all(torch.equal(j.out, o) for j, o in zip(jobs, outs))
    moved = sum(j.bytes_moved() for j in jobs)
    cpu = None
    lib, name = _ref_library()
    if cpu_budget > 0 and lib.exists():
        # the reference library's one-op-per-call path over the first jobs of the same list,
        # one host core, each output compared with the GPU work list's
        from vfhe_b200.native import Engine
        from vfhe_b200.worklist import run_job_on_engine

        ref = Engine(lib)
        done, same, t0 = 0, True, time.perf_counter()
        for j in jobs:
            got = run_job_on_engine(ref, j)
            same = same and bool(np.array_equal(got, j.out.cpu().numpy().view(np.uint64).reshape(got.shape)))
            done += 1
            if time.perf_counter() - t0 > cpu_budget:
                break
        el = time.perf_counter() - t0
        cpu = {"jobs_per_s": done / el, "cores": 1, "kind": "reference", "bit_exact_vs_work_list": same,
               "sample": f"the first {done} of the {len(jobs)} jobs, one at a time through the reference's "
                         f"{name} engine's cdef calls, one thread, {el:.1f} s"}
    res = {
        "jobs": count, "jobs_per_s": count / (ms_wl * 1e-3), "ms_per_run": ms_wl,
        "per_call_jobs_per_s": count / (ms_pc * 1e-3), "per_call_ms": ms_pc, "per_call_calls": calls,
        "speedup_vs_per_call": ms_pc / ms_wl, "bit_exact_vs_per_call": bool(exact),
        "kernels_per_run": wl.launches, "persistent": wl.persistent, "phase_ms_last_run": phases,
        "graph_of_pool_launches": {"jobs_per_s": count / (ms_graph * 1e-3), "ms_per_run": ms_graph,
                                   "kernels_per_run": graph_launches, "bit_exact_vs_persistent": bool(persistent_exact)},
        "device_bytes": wl.device_bytes,
        "algorithmic_gb_per_s": moved / (ms_wl * 1e-3) / 1e9,
        "mix": {"chain": sum(j.kind == "chain" for j in jobs), "keyswitch": sum(j.kind == "keyswitch" for j in jobs)},
    }
    if cpu is not None:
        res["cpu_reference"] = cpu
    wl.close()
    del jobs, outs, ws
    torch.cuda.empty_cache()
    return res


def _balanced_digits(c: np.ndarray, base_log: int, levels: int) -> np.ndarray:
    """Signed gadget digits of 32-bit torus values: round to base_log * levels bits, then
    digits in [-B/2, B/2) from the least significant up with a carry (the decomposition
    the FFT external product applies).  Returns [levels][...] int64, most significant
    digit first."""
    total = base_log * levels
    r = ((c.astype(np.uint64) + (1 << (31 - total))) >> (32 - total)) & ((1 << total) - 1)
    r = r.astype(np.int64)
    half, full = 1 << (base_log - 1), 1 << base_log
    out = np.zeros((levels,) + c.shape, dtype=np.int64)
    for lvl in range(levels - 1, -1, -1):
        d = r & (full - 1)
        r >>= base_log
        carry = d >= half
        d = np.where(carry, d - full, d)
        r = r + carry
        out[lvl] = d
    return out


def fft_product_error(eng, keys, dev, p, count: int = 8) -> dict:
    """Max absolute error of the GPU's FP64-FFT external product (GLWE x GGSW(s_0)) against
    the exact integer negacyclic product, computed here in int64 (every partial sum of
    digit x 32-bit key coefficient products stays below 2^52), over `count` random GLWE
    ciphertexts; errors are distances on the 2^32 torus."""
    import torch

    from vfhe_b200.cggi_fft import to_device, to_host

    N, lv, bl = p.N, p.bs_levels, p.bs_base_log
    rng = np.random.default_rng(SEED + 31)
    c = rng.integers(0, 1 << 32, (count, 2 * N), dtype=np.uint64).astype(np.uint32)
    out = torch.empty((count, 2 * N), dtype=torch.int32, device="cuda")
    frac = torch.empty(count, dtype=torch.float64, device="cuda")
    ffi = eng.ffi
    dc = to_device(c)
    rc = eng.lib.vfhe_cuda_cggi_fft_external_product(
        ffi.cast("uint32_t*", out.data_ptr()), ffi.cast("uint32_t*", dc.data_ptr()), count,
        ffi.cast("double*", dev.bsk_f[: 2 * lv * 2].data_ptr()), N, bl, lv, ffi.cast("double*", frac.data_ptr()),
        ffi.cast("void*", torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    got = to_host(out).astype(np.uint32).astype(np.int64)
    ggsw = np.asarray(keys.bsk[0], dtype=np.uint32).astype(np.int64).reshape(2 * lv, 2, N)
    worst = 0
    for b in range(count):
        dig = _balanced_digits(c[b].reshape(2, N), bl, lv)  # [lv][comp][N]
        exact = np.zeros((2, N), dtype=np.int64)
        for comp in range(2):
            for lvl in range(lv):
                row = comp * lv + lvl
                for oc in range(2):
                    full = np.convolve(dig[lvl, comp], ggsw[row, oc])
                    exact[oc] += full[:N]
                    exact[oc, : N - 1] -= full[N:]
        diff = (got[b].reshape(2, N) - exact) & 0xFFFFFFFF
        dist = np.minimum(diff, (1 << 32) - diff)
        worst = max(worst, int(dist.max()))
    return {"max_abs_error": worst, "unit": "torus units (2^-32)", "products": count,
            "max_rounding_fraction": float(frac.max()),
            "reference": "exact integer negacyclic product (int64), same signed digits"}


def cggi_fft_leg(eng, count: int, reps: int, million: bool = False) -> dict:
    """Torus CGGI programmable bootstrap (n = 630, N = 1024, base 2^7 x 3, key switch
    2^2 x 8): `count` LWEs of random 4-bit messages through one seeded 16-entry table
    per batch; bootstraps/s, LUT mismatches and phase error (torus fractions)."""
    import torch

    from vfhe_b200.cggi_fft import CggiFft, TorusKeys, TorusParams, test_vector, to_device, to_host

    p = TorusParams()
    rng = np.random.default_rng(SEED + 9)
    keys = TorusKeys.generate(p, rng)
    dev = CggiFft(keys, eng)
    lut = rng.integers(0, p.t, p.t)
    tv = to_device(test_vector(lut, p))
    m = rng.integers(0, p.t, count)
    lwe = to_device(keys.encrypt(m, rng))
    dev.bootstrap(lwe[:256], tv)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    profile_range(None, "cggi_fft", True)
    ev[0].record(stream)
    for _ in range(reps):
        ext = dev.blind_rotate(lwe, tv)
    ev[1].record(stream)
    for _ in range(reps):
        out = dev.keyswitch(ext)
    ev[2].record(stream)
    torch.cuda.synchronize()
    profile_range(None, "cggi_fft", False)
    br_ms = ev[0].elapsed_time(ev[1]) / reps
    ks_ms = ev[1].elapsed_time(ev[2]) / reps
    res_host, ext_host = to_host(out), to_host(ext)
    err = np.abs(keys.phases(res_host) - lut[m] * p.delta) / 2.0**32
    err_ext = np.abs(keys.phases(ext_host, keys.S) - lut[m] * p.delta) / 2.0**32
    res = {
        "workload": f"{count} LWEs, n=630 binary key sigma 2^-15; GLWE N=1024 k=1 binary key sigma 2^-25; "
                    "gadget 2^7 x 3; key switch 2^2 x 8 (key noise sigma 2^-15); 4-bit messages + padding, "
                    "16-entry LUT",
        "bootstraps_per_s": count / ((br_ms + ks_ms) * 1e-3), "blind_rotation_ms": br_ms, "keyswitch_ms": ks_ms,
        "checked": count, "box_half_width": 0.5 / (2 * p.t),
        # after blind rotation + extraction (key S): the bootstrap's own noise
        "mismatches_extracted": int((keys.decrypt(ext_host, keys.S) != lut[m]).sum()),
        "phase_error_extracted_mean": float(err_ext.mean()), "phase_error_extracted_max": float(err_ext.max()),
        # after the key switch back to s: adds the key-switching key's noise
        "mismatches": int((keys.decrypt(res_host) != lut[m]).sum()),
        "phase_error_mean": float(err.mean()), "phase_error_max": float(err.max()),
    }
    res["fft_external_product"] = fft_product_error(eng, keys, dev, p)
    if million:
        total, bad, bad_ext, worst, worst_ext = 0, 0, 0, 0.0, 0.0
        mc = 16384  # LWEs per batch of the 10^6 run
        while total < 1_000_000:
            mm = rng.integers(0, p.t, mc)
            e = dev.blind_rotate(to_device(keys.encrypt(mm, rng)), tv)
            o, eh = to_host(dev.keyswitch(e)), to_host(e)
            bad += int((keys.decrypt(o) != lut[mm]).sum())
            bad_ext += int((keys.decrypt(eh, keys.S) != lut[mm]).sum())
            worst = max(worst, float((np.abs(keys.phases(o) - lut[mm] * p.delta) / 2.0**32).max()))
            worst_ext = max(worst_ext, float((np.abs(keys.phases(eh, keys.S) - lut[mm] * p.delta) / 2.0**32).max()))
            total += mc
        res["million"] = {"bootstraps": total, "mismatches_extracted": bad_ext, "phase_error_extracted_max": worst_ext,
                          "mismatches": bad, "phase_error_max": worst,
                          "note": "mismatches_extracted counts the bootstrapped LWEs (blind rotation + sample "
                                  "extraction, the reference's functional_bootstrap); mismatches adds the LWE key "
                                  "switch back to n = 630, whose key carries the LWE noise sigma 2^-15"}
    del dev
    torch.cuda.empty_cache()
    return res


def _rns_cggi_setup(engine, n_lwe: int, count: int, seed: int):
    """The reference's CGGI16 (RNS gadget) at N = 1024, [50, 50, 50] (one special), a
    binary LWE key of dimension n_lwe, 5-bit LUT precision: keys and LWEs (seeded)."""
    from vfhe_b200.arith import Ring
    from vfhe_b200.fhe import CGGI16
    from vfhe_b200.mlwe import LWE_Key, MLWE_Scheme, encrypt_lwe
    from vfhe_b200.native import use_engine

    with use_engine(engine):
        rng = np.random.default_rng(seed)
        Rq = Ring(1024, prime_size=[50, 50, 50], split_degree=1)
        in_ring = Rq.quotient_ring(ell=2)
        s = MLWE_Scheme(Rq, special_primes=1, module_rank=1, max_lvl=1)
        key_s = [int(v) for v in rng.integers(0, 2, n_lwe)]
        out_key = s.key_gen_sparse(64, 3.2, ternary=False, rng=rng)
        cg = CGGI16(s)
        bk = cg.generate_bootstrap_key(LWE_Key(ring=in_ring, key=key_s, n=n_lwe), out_key, rng=rng)
        t = 16
        lut = [int(v) for v in rng.integers(0, t, t)]
        tv = cg.LUT_packing(lut, t, 5)
        msgs = [int(v) for v in rng.integers(0, t, count)]
        lwes = [encrypt_lwe(in_ring, key_s, [round(m * in_ring.q_l / 32) % q for q in in_ring.primes], 3.2, rng)
                for m in msgs]
        ok = out_key.extract_lwe_key()
        key2 = LWE_Key(ring=in_ring, key=ok.get_s(), n=ok.n)
        return s, cg, bk, tv, lwes, msgs, lut, in_ring, key2


def rns_cggi_leg(eng, count: int = 1024, cpu_bootstraps: int = 2) -> dict:
    """Batched RNS CGGI16 (the reference's scheme) at n = 630, N = 1024 on the GPU, and
    the reference library's own functional_bootstrap on one host core."""
    import torch

    from vfhe_b200.batch import CggiBatch, bootstrap_key_tensor, to_device, to_host
    from vfhe_b200.mlwe import LWE

    s, cg, bk, tv, lwes, msgs, lut, in_ring, key2 = _rns_cggi_setup(eng, 630, count, SEED + 11)
    a = to_device(np.stack([np.array(x.get_a(), dtype=np.uint64) for x in lwes]))
    b = to_device(np.stack([np.array(x.get_b(), dtype=np.uint64) for x in lwes]))
    tv.to_coeff()
    tvt = to_device(np.stack([tv.component_rows(0), tv.component_rows(1)]))
    bkt = bootstrap_key_tensor(bk)
    runner = CggiBatch(s, eng)
    oa, ob = runner.bootstrap(a, b, bkt, tvt, 16)  # captures the blind-rotation graph
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    profile_range(None, "cggi_rns", True)
    e0.record(stream)
    oa, ob = runner.bootstrap(a, b, bkt, tvt, 16)
    e1.record(stream)
    torch.cuda.synchronize()
    profile_range(None, "cggi_rns", False)
    ms = e0.elapsed_time(e1)
    ha, hb = to_host(oa), to_host(ob)
    def phase_error(ph: int, want: int, q: int) -> float:
        """Distance of a phase from want * q / 32 on the ring Z_q, as a fraction of q."""
        d = (ph - round(want * q / 32)) % q
        return min(d, q - d) / q

    bad, errs = 0, []
    for i in range(min(count, 64)):
        o = LWE(ring=in_ring, n=1024)
        o.set_rows(ha[i], hb[i])
        ph = o.phase(key2, recompose=True)
        bad += int(round(ph * 32 / in_ring.q_l) % 32 != lut[msgs[i]])
        errs.append(phase_error(ph, lut[msgs[i]], in_ring.q_l))
    res = {"workload": f"{count} LWEs, n=630, N=1024, RNS gadget over 2 x 50-bit primes + 1 special, 16-entry LUT",
           "gpu_bootstraps_per_s": count / (ms * 1e-3), "gpu_ms": ms, "checked": min(count, 64),
           "mismatches": bad, "phase_error_mean": float(np.mean(errs)), "phase_error_max": float(np.max(errs)),
           "phase_error_unit": "fraction of Q (half box = 1/64)"}
    lib, name = _ref_library()
    if lib.exists() and cpu_bootstraps > 0:
        from vfhe_b200.native import Engine

        ref = Engine(lib)
        rs, rcg, rbk, rtv, rlwes, rmsgs, rlut, rin, rkey2 = _rns_cggi_setup(ref, 630, cpu_bootstraps, SEED + 12)
        routs = [LWE(ring=rin) for _ in rlwes]
        t0 = time.perf_counter()
        for x, o in zip(rlwes, routs):
            rcg.functional_bootstrap(o, rtv, x, rbk, torus_base=16)
        res["cpu_reference_ms_per_bootstrap"] = 1e3 * (time.perf_counter() - t0) / cpu_bootstraps
        rerr = [phase_error(o.phase(rkey2, recompose=True), rlut[m], rin.q_l) for o, m in zip(routs, rmsgs)]
        res["cpu_reference_phase_error_max"] = float(np.max(rerr))
        res["cpu_reference"] = f"reference's {name} engine, one core, {cpu_bootstraps} bootstraps"
    return res


def ntt_round_trip_leg(eng, reps: int = 20, cpu_budget: float = 3.0, pool=None) -> dict:
    """The plain RNS NTT round trip: 64 pairs (a, b) in Z_q[X]/(X^4096 + 1), L = 3 (the
    three largest 50-bit NTT primes of the reference's generator for the split), uniform
    residues; forward NTT of both, the incomplete product with the split twist, inverse
    NTT -- one vfhe_cuda_ntt_mul_intt_batch call per step.  Reported at the reference's
    default split (4, P = 1024) and at split 1.  Device-resident steps flush L2 first
    (the working set, 18.9 MB, would otherwise stay in the 126 MB L2); the e2e figure
    copies the pinned host inputs in and the products out inside every step.  The
    reference's own library times the same chain (polynomial_RNSc_to_RNS x 2,
    polynomial_mul_RNS_polynomial, polynomial_RNS_to_RNSc; rns_polynomial.c:311-356,
    582-614) on one host core."""
    import torch

    from vfhe_b200.arith import Ring
    from vfhe_b200.batch import to_device
    from vfhe_b200.native import Engine

    pairs, N, L = 64, 4096, 3
    ffi = eng.ffi
    stream = torch.cuda.current_stream()
    sp = ffi.cast("void*", stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    peak, _ = measured_peaks()
    alg_bytes = pairs * L * N * 8 * 3
    res = {"workload": "64 pairs, N=4096, L=3 (50-bit primes), NTT -> product -> INTT per pair",
           "algorithmic_bytes_per_step": alg_bytes}
    lib, name = _ref_library()
    ref = Engine(lib) if lib.exists() else None
    for split in (None, 1):
        R = Ring(N, prime_size=[50] * L, split_degree=split, engine=eng)
        rng = np.random.default_rng(SEED + 21)
        ha = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in R.primes]) for _ in range(pairs)])
        hb = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in R.primes]) for _ in range(pairs)])
        a, b = to_device(ha), to_device(hb)
        out = torch.empty_like(a)
        limbs = ffi.new("uint32_t[]", R.prime_indices)
        pa, pb, po = (ffi.cast("uint64_t*", t.data_ptr()) for t in (a, b, out))

        def call():
            if eng.lib.vfhe_cuda_ntt_mul_intt_batch(R.NTT, po, pa, pb, pairs, limbs, L, sp) != 0:
                eng.check("ntt_mul_intt_batch")

        for _ in range(3):
            call()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        leg = "roundtrip" if split is None else "roundtrip_split1"
        profile_range(None, leg, True)
        for e0, e1 in evs:
            flush.zero_()
            e0.record(stream)
            call()
            e1.record(stream)
        torch.cuda.synchronize()
        profile_range(None, leg, False)
        ms = sum(e0.elapsed_time(e1) for e0, e1 in evs) / reps
        # end to end from pinned host buffers
        hA = torch.from_numpy(ha.view(np.int64)).pin_memory()
        hB = torch.from_numpy(hb.view(np.int64)).pin_memory()
        hO = torch.empty(out.shape, dtype=torch.int64).pin_memory()
        for e0, e1 in evs:
            e0.record(stream)
            a.copy_(hA, non_blocking=True)
            b.copy_(hB, non_blocking=True)
            call()
            hO.copy_(out, non_blocking=True)
            e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = sum(e0.elapsed_time(e1) for e0, e1 in evs) / reps
        key = f"split{R.split_degree}"
        res[key] = {"pairs_per_s": pairs / (ms * 1e-3), "ms_per_step": ms,
                    "frac_hbm": alg_bytes / (ms * 1e-3) / 1e9 / peak, "l2": "flushed before every step",
                    "e2e": {"pairs_per_s": pairs / (e2e_ms * 1e-3), "ms_per_step": e2e_ms,
                            "h2d_bytes_per_step": int(ha.nbytes + hb.nbytes), "d2h_bytes_per_step": int(ha.nbytes)}}
        if ref is not None:
            Rr = Ring(N, prime_size=[50] * L, split_degree=split, engine=ref)
            assert Rr.primes == R.primes
            from vfhe_b200.arith import Polynomial

            P = [Polynomial(Rr) for _ in range(5)]
            P[0].set_rows(ha[0])
            P[1].set_rows(hb[0])
            for x in P[:2]:
                x.rns_mask = Rr.mask
            rl = ref.lib
            done, t0 = 0, time.perf_counter()
            while time.perf_counter() - t0 < cpu_budget:
                rl.polynomial_RNSc_to_RNS(P[2].obj, P[0].obj)
                rl.polynomial_RNSc_to_RNS(P[3].obj, P[1].obj)
                rl.polynomial_mul_RNS_polynomial(P[4].obj, P[2].obj, P[3].obj)
                rl.polynomial_RNS_to_RNSc(P[4].obj, P[4].obj)
                done += 1
            el = time.perf_counter() - t0
            res[key]["cpu_reference"] = {"pairs_per_s": done / el, "cores": 1, "kind": "reference",
                                         "sample": f"{done} pairs on the reference's {name} engine, one thread"}
            if pool is not None:
                allc = pool.rate(_cpu_roundtrip_worker, (split, cpu_budget), SEED + 40)
                res[key]["cpu_reference_all_cores"] = {
                    "pairs_per_s": allc["value"], "cores": allc["cores"], "kind": "reference",
                    "sample": f"one process per host core, {cpu_budget:.0f} s of chains each, the reference's "
                              f"{allc['engine']} engine"}
        del a, b, out
    del flush
    return res


def composed_leg(eng, reps: int = 3) -> dict:
    """The operations built by composing the engine's calls, timed through the cdef on the
    cuda engine and on the reference's own library (one host core), same inputs:
    mlwe_trace (mlwe.c:436-444: log2 N automorphism key switches) at N = 4096,
    mlwe_full_packing_keyswitch (mlwe.c:343-430) of 16 LWEs at N = 1024, and the CKKS
    rational rescale (ckks.py:150-202) of a ciphertext between levels sharing two primes
    at N = 4096.  Random residues stand in for keys and ciphertexts (the calls are exact
    modular arithmetic).  Per call: host-addressable rows in, results readable on return."""
    from vfhe_b200.arith import Ring, reset_registries
    from vfhe_b200.arith import repr as prepr
    from vfhe_b200.fhe import CKKS_Ciphertext, CKKS_Scheme
    from vfhe_b200.mlwe import LWE, MLWE, MLWE_Scheme, MLWE_Set
    from vfhe_b200.native import Engine, use_engine

    lib, name = _ref_library()
    engines = [("cuda", eng)] + ([("reference", Engine(lib))] if lib.exists() else [])
    rng = np.random.default_rng(SEED + 60)

    def rows(primes, N):
        return np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in primes])

    def mlwe(s, ring, r0, r1, rep):
        m = MLWE(s, ring=ring) if ring is not None else MLWE(s, lvl=0)
        m.set_component_rows(0, r0)
        m.set_component_rows(1, r1)
        m.repr = rep
        return m

    def timed(fn):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        return 1e3 * (time.perf_counter() - t0) / reps

    res = {}
    # trace at N = 4096 (12 automorphism key switches)
    N, logN = 4096, 12
    base = Ring(N, prime_size=[50, 50, 50], split_degree=1, engine=eng)
    primes = base.primes
    ct = [rows(primes[:2], N) for _ in range(2)]
    keys = [[[rows(primes, N) for _ in range(2)] for _ in range(2)] for _ in range(logN)]
    out = {}
    for tag, e in engines:
        reset_registries()
        with use_engine(e):
            R = Ring(N, prime_size=[50, 50, 50], primes=primes, split_degree=1, engine=e)
            s = MLWE_Scheme(R, special_primes=1, module_rank=1, max_lvl=1)
            c = mlwe(s, None, ct[0], ct[1], prepr.coeff)
            sets = [MLWE_Set([[mlwe(s, s.special_rings[0], k[d][0], k[d][1], prepr.ntt) for d in range(2)]])
                    for k in keys]
            ksks = MLWE_Set.flatten_array(sets)
            o = MLWE(s, lvl=0)
            out[tag] = timed(lambda: R.lib.mlwe_trace(o.obj, c.obj, ksks.obj, 0))
            e.check("mlwe_trace")
    res["trace_n4096"] = out
    # full packing key switch of 16 LWEs at N = 1024
    N, size = 1024, 16
    base = Ring(N, prime_size=[50, 50, 50], split_degree=1, engine=eng)
    primes = base.primes
    lwe_rows = [(rows(primes[:2], N), [int(rng.integers(0, q)) for q in primes[:2]]) for _ in range(size)]
    krows = [[rows(primes, N) for _ in range(2)] for _ in range(2 * N)]
    out = {}
    for tag, e in engines:
        reset_registries()
        with use_engine(e):
            R = Ring(N, prime_size=[50, 50, 50], primes=primes, split_degree=1, engine=e)
            s = MLWE_Scheme(R, special_primes=1, module_rank=1, max_lvl=1)
            lwes = []
            for a, b in lwe_rows:
                x = LWE(s.rings[0], n=N)
                x.set_rows(a, b)
                lwes.append(x)
            ksk = MLWE_Set([[mlwe(s, s.special_rings[0], krows[2 * i + d][0], krows[2 * i + d][1], prepr.ntt)
                             for d in range(2)] for i in range(N)])
            o = MLWE(s, lvl=0)
            arr = R.ffi.new("void*[]", [x.obj for x in lwes])
            out[tag] = timed(lambda: R.lib.mlwe_full_packing_keyswitch(o.obj, arr, size, ksk.obj, 0))
            e.check("mlwe_full_packing_keyswitch")
    res["full_packing_keyswitch_16_n1024"] = out
    # rational rescale between levels sharing two primes, N = 4096
    N = 4096
    base = Ring(N, split_degree=1, prime_size=[50, 50, 50, 30, 50], engine=eng)
    primes = base.primes
    ct = None
    out = {}
    for tag, e in engines:
        reset_registries()
        with use_engine(e):
            Rq = Ring(N, split_degree=1, prime_size=[50, 50, 50, 30, 50], primes=primes, engine=e)
            sub = lambda *ix: Rq.quotient_ring(mask=sum(1 << Rq.prime_indices[i] for i in ix))  # noqa: E731
            s = CKKS_Scheme([sub(0, 1, 2), sub(0, 1, 3)], scaling_factor=2**50, special_primes=1,
                            special_rings=[sub(0, 1, 2, 4), sub(0, 1, 3, 4)])
            if ct is None:
                ct = [rows(s.rings[0].primes, N) for _ in range(2)]
            c = CKKS_Ciphertext(s, lvl=0)
            c.set_component_rows(0, ct[0])
            c.set_component_rows(1, ct[1])
            c.repr = prepr.coeff
            out[tag] = timed(lambda: s.rational_rescale(c))
            e.check("rational_rescale")
    res["rational_rescale_n4096"] = out
    reset_registries()
    for v in res.values():
        v["unit"] = "ms per call"
        if "reference" in v:
            v["reference"] = {"ms": v["reference"], "cores": 1, "engine": name}
    return res


def encrypt_leg(eng, s, key, msgs, reps: int = 5, cpu_encryptions: int = 8) -> dict:
    """Batched CKKS encryption (vfhe_cuda_rlwe_encrypt_batch) of the workload's batch of
    coefficient-domain plaintexts at N = 2^14, L = 9, and the reference library's own
    CKKS_Scheme.encrypt (mlwe_RNSc_sample) on one host core."""
    import torch

    from vfhe_b200.batch import CkksBatch

    enc = CkksBatch(s.rings[0], s.special_rings[0].prime_indices[-1], eng)
    out = enc.encrypt(key, msgs)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    profile_range(None, "encrypt", True)
    e0.record(stream)
    for _ in range(reps):
        enc.encrypt(key, msgs, out=out)
    e1.record(stream)
    torch.cuda.synchronize()
    profile_range(None, "encrypt", False)
    ms = e0.elapsed_time(e1) / reps
    B = msgs.shape[0]
    res = {"workload": f"{B} ciphertexts, N=2^14, L=9, ternary key, sigma 3.2, ChaCha20 randomness",
           "ciphertexts_per_s": B / (ms * 1e-3), "ms_per_batch": ms}
    lib, name = _ref_library()
    if lib.exists() and cpu_encryptions > 0:
        from vfhe_b200.native import Engine

        from vfhe_b200.arith import Ring
        from vfhe_b200.fhe import CKKS_Scheme
        from vfhe_b200.native import use_engine

        ref = Engine(lib)
        with use_engine(ref):
            rs = CKKS_Scheme(Ring(N_DEG, prime_size=PRIME_SIZES, split_degree=1), scaling_factor=SCALE,
                             special_primes=1)
            rkey = rs.key_gen_uniform_ternary(3.2, np.random.default_rng(SEED + 13))
            pt = rs.encode([0.5] * (N_DEG // 2))
            t0 = time.perf_counter()
            for _ in range(cpu_encryptions):
                rs.encrypt(pt, rkey)
            res["cpu_reference_ms_per_ciphertext"] = 1e3 * (time.perf_counter() - t0) / cpu_encryptions
        res["cpu_reference"] = f"reference's {name} engine, one core, {cpu_encryptions} encryptions"
    return res


def serving_leg(eng, requests: int, rates=(50.0, 200.0, 1000.0)) -> dict:
    """Poisson request streams of mixed CKKS (N 2^13..2^16, L 4..24: multiply+relin+
    rescale or rotate) and CGGI16 bootstrap batches (1..1024 LWEs, n = 630, N = 1024),
    keys and ciphertexts resident in HBM, 160 GB budget: continuous batching (64 per
    batch, 4 streams) vs the plain path (one request per call, one stream), p50/p99 and
    throughput per arrival rate; plus CKKS multiply saturation at N = 2^14, L = 9."""
    import torch

    from vfhe_b200.serve import Server, ServingMix, poisson_arrivals, run_stream

    mix = ServingMix(eng, seed=SEED + 5)
    budget = 160 * 10**9
    out = {"budget_bytes": budget, "resident_bytes": mix.resident, "requests_per_rate": requests,
           "mix": "90% CKKS (half mul+relin+rescale, half rotate) over (2^13,4),(2^14,9),(2^15,16),(2^16,24); "
                  "10% CGGI16 programmable bootstraps, batches of 1..1024 LWEs (log-uniform), n=630, N=1024, "
                  "gadget 2^7 x 3, key switch 2^2 x 8 (torus FP64-FFT path)",
           "rates": []}
    reqs = mix.requests(requests, seed=SEED + 6, ckks_share=0.9)
    p = mix.ckks[1]
    sat = [("mul", 1, i % len(p.cts), (i + 1) % len(p.cts)) for i in range(256)]
    modes = {"served": (4, 64), "plain": (1, 1)}
    servers = {}
    for name, (streams, mb) in modes.items():
        srv = Server(budget, streams=streams, max_batch=mb, engine=eng)
        mix.register(srv)
        srv.reserve(16 * 10**9 if mb > 1 else 2 * 10**9)
        # warm-up: every CGGI batch-size bucket once, a short mixed stream and a short
        # multiply burst
        for k in range(11):
            run_stream(mix, srv, [("cggi", -1, 1 << k, 0)], np.zeros(1))
        run_stream(mix, srv, reqs[:24], np.zeros(24))
        run_stream(mix, srv, sat[:128], np.zeros(128))
        servers[name] = srv
    for rate in rates:
        arr = poisson_arrivals(rate, len(reqs), np.random.default_rng(int(rate)))
        row = {"rate_rps": rate}
        for name, srv in servers.items():
            b0 = srv.stats()["batches"]
            r = run_stream(mix, srv, reqs, arr)
            row[name] = {k: r[k] for k in ("p50_ms", "p99_ms", "mean_ms", "throughput_rps")}
            row[name]["batches"] = int(srv.stats()["batches"] - b0)
        out["rates"].append(row)
    # saturation: 256 CKKS multiplies at the benchmark's parameters, all queued at t = 0
    res = {}
    for name, srv in servers.items():
        b0 = srv.stats()["batches"]
        r = run_stream(mix, srv, sat, np.zeros(len(sat)))
        res[name] = {k: r[k] for k in ("p50_ms", "p99_ms", "throughput_rps")}
        res[name]["batches"] = int(srv.stats()["batches"] - b0)
    for srv in servers.values():
        srv.close()
    res["speedup"] = res["served"]["throughput_rps"] / res["plain"]["throughput_rps"]
    out["ckks_mul_saturation_n2p14_L9"] = res
    del mix
    torch.cuda.empty_cache()
    return out


def run_cuda_arm(args) -> None:
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        os.environ.setdefault("VFHE_CUDA_DEVICE", str(local))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from vfhe_b200.batch import CkksBatch, ciphertext_rows, key_tensor, to_device
    from vfhe_b200.native import cuda_engine

    eng = cuda_engine()
    for spec in args.ntt_schedule:
        lp, rest = spec.split(":")
        sched = [int(v) for v in rest.split(",")]
        for bucket in range(32):
            if eng.lib.vfhe_cuda_ntt_set_schedule(int(lp), bucket, *sched) != 0:
                raise SystemExit(f"--ntt-schedule {spec}: refused by the engine")
    PAIRS = args.pairs  # noqa: N806  (the workload's batch; 256 unless profiling a small case)
    share = pair_share(rank, PAIRS)
    s, key, rlk, gks, rot_steps, zs, cts = build_workload(eng, PAIRS, SEED, first_pair=share.start)
    for c in cts:
        c.to_NTT()
    host1 = np.stack([ciphertext_rows(c) for c in cts[0::2]])
    host2 = np.stack([ciphertext_rows(c) for c in cts[1::2]])
    d1, d2 = to_device(host1), to_device(host2)
    rlk_t = key_tensor(rlk)
    gk_t = {k: key_tensor(v) for k, v in gks.items()}
    special = s.special_rings[0].prime_indices[-1]
    mul = CkksBatch(s.rings[0], special, eng)
    rotb = CkksBatch(s.rings[1], special, eng)
    gens = [s.galois_gen(k) for k in rot_steps]
    keys = [gk_t[k] for k in rot_steps]
    prod = torch.empty((PAIRS, 2, 8, N_DEG), dtype=torch.int64, device="cuda")
    rot = torch.empty_like(prod)
    stream = torch.cuda.current_stream()

    def step():
        mul.mul_relin_rescale(d1, d2, rlk_t, out=prod)
        rotb.rotate(prod, gens, keys, out=rot)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()

    # ---- device-resident throughput
    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    launches0 = eng.lib.vfhe_cuda_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier()
        # the timed region is also the profiler's capture range (ncu --profile-from-start off)
        profile_range(args, "ckks", True)
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        barrier()
        profile_range(args, "ckks", False)
    launches = eng.lib.vfhe_cuda_launch_count() - launches0
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist, "cuda")
    value = whole_job_rate(PAIRS, world, ms)

    # ---- end to end: pinned host inputs in, host results out, every step.  Steps are
    # pipelined over two buffer sets and three streams (copy in, compute, copy out), as
    # a caller of the batched API would run them: step i's inputs travel while step i-1
    # computes and step i-2's results travel back.  The headline figure moves the
    # ciphertexts in the compact wire format (WireFormat: each residue at its prime's
    # bit length, unpacked and packed on the GPU inside the step); the plain uint64
    # transport is timed beside it.
    from vfhe_b200.batch import WireFormat

    wf_in = WireFormat.for_ring(s.rings[0], engine=eng)
    wf_out = WireFormat.for_ring(s.rings[1], engine=eng)
    h1 = torch.from_numpy(host1.view(np.int64)).pin_memory()
    h2 = torch.from_numpy(host2.view(np.int64)).pin_memory()
    h1p = wf_in.pack(d1).cpu().pin_memory()
    h2p = wf_in.pack(d2).cpu().pin_memory()
    torch.cuda.synchronize()
    hout = [torch.empty(rot.shape, dtype=torch.int64).pin_memory() for _ in range(2)]
    houtp = [torch.empty((PAIRS, wf_out.item_bytes), dtype=torch.uint8).pin_memory() for _ in range(2)]
    din = [(d1, d2), (torch.empty_like(d1), torch.empty_like(d2))]
    dinp = [(torch.empty_like(h1p, device="cuda"), torch.empty_like(h2p, device="cuda")) for _ in range(2)]
    doutp = [torch.empty_like(houtp[0], device="cuda") for _ in range(2)]
    dprod = [prod, torch.empty_like(prod)]
    drot = [rot, torch.empty_like(rot)]
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_comp = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    e2e_steps = max(4, min(args.steps, 10))

    def e2e_run(count, packed):
        for i in range(count):
            b = i % 2
            a1, a2 = din[b]
            src1, src2 = (dinp[b] if packed else din[b])
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_comp[b])  # step i-2 has finished reading these inputs
                src1.copy_(h1p if packed else h1, non_blocking=True)
                src2.copy_(h2p if packed else h2, non_blocking=True)
                ev_in[b].record(s_in)
            stream.wait_event(ev_in[b])
            if i >= 2:
                stream.wait_event(ev_out[b])  # step i-2's results have left drot[b] / doutp[b]
            if packed:
                wf_in.unpack(src1, a1.shape, out=a1, stream=stream)
                wf_in.unpack(src2, a2.shape, out=a2, stream=stream)
            mul.mul_relin_rescale(a1, a2, rlk_t, out=dprod[b], stream=stream)
            rotb.rotate(dprod[b], gens, keys, out=drot[b], stream=stream)
            if packed:
                wf_out.pack(drot[b], out=doutp[b], stream=stream)
            ev_comp[b].record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_comp[b])
                if packed:
                    houtp[b].copy_(doutp[b], non_blocking=True)
                else:
                    hout[b].copy_(drot[b], non_blocking=True)
                ev_out[b].record(s_out)
        stream.wait_stream(s_out)

    def e2e_time(packed):
        e2e_run(2, packed)
        barrier()
        ev0.record(stream)
        e2e_run(e2e_steps, packed)
        ev1.record(stream)
        barrier()
        return max_over_ranks(ev0.elapsed_time(ev1) / e2e_steps, dist, "cuda")

    e2e_ms_plain = e2e_time(False)
    e2e_value_plain = whole_job_rate(PAIRS, world, e2e_ms_plain)
    e2e_ms = e2e_time(True)
    e2e_value = whole_job_rate(PAIRS, world, e2e_ms)

    # the wire format with the sender's packing and the receiver's unpacking on the host
    # inside the timed region (vfhe_cuda_pack_rows_host / _unpack_rows_host on every host
    # thread): step i's inputs are packed while the GPU works on step i-1, and step i-1's
    # results are unpacked into uint64 rows after step i is enqueued.  Host wall clock.
    host_threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    h1n, h2n = h1.numpy(), h2.numpy()
    hpk = [(torch.empty_like(h1p).pin_memory(), torch.empty_like(h2p).pin_memory()) for _ in range(2)]
    res_rows = np.empty(tuple(rot.shape), dtype=np.int64)

    def e2e_hostpack_run(count):
        for i in range(count):
            b = i % 2
            if i >= 2:
                ev_in[b].synchronize()  # step i-2's copy from these packed buffers is done
            wf_in.pack_host(h1n, out=hpk[b][0].numpy(), nthreads=host_threads)
            wf_in.pack_host(h2n, out=hpk[b][1].numpy(), nthreads=host_threads)
            a1, a2 = din[b]
            src1, src2 = dinp[b]
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_comp[b])
                src1.copy_(hpk[b][0], non_blocking=True)
                src2.copy_(hpk[b][1], non_blocking=True)
                ev_in[b].record(s_in)
            stream.wait_event(ev_in[b])
            if i >= 2:
                stream.wait_event(ev_out[b])
            wf_in.unpack(src1, a1.shape, out=a1, stream=stream)
            wf_in.unpack(src2, a2.shape, out=a2, stream=stream)
            mul.mul_relin_rescale(a1, a2, rlk_t, out=dprod[b], stream=stream)
            rotb.rotate(dprod[b], gens, keys, out=drot[b], stream=stream)
            wf_out.pack(drot[b], out=doutp[b], stream=stream)
            ev_comp[b].record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_comp[b])
                houtp[b].copy_(doutp[b], non_blocking=True)
                ev_out[b].record(s_out)
            if i >= 1:
                ev_out[1 - b].synchronize()
                wf_out.unpack_host(houtp[1 - b].numpy(), res_rows, nthreads=host_threads)
        ev_out[(count - 1) % 2].synchronize()
        wf_out.unpack_host(houtp[(count - 1) % 2].numpy(), res_rows, nthreads=host_threads)

    e2e_hostpack_run(2)
    barrier()
    t0 = time.perf_counter()
    e2e_hostpack_run(e2e_steps)
    barrier()
    e2e_ms_hostpack = max_over_ranks(1e3 * (time.perf_counter() - t0) / e2e_steps, dist, "cuda")
    hostpack_ok = bool(np.array_equal(res_rows, drot[(e2e_steps - 1) % 2].cpu().numpy()))
    # the packed transport delivers the same results: compare the last step's output
    hres = torch.empty_like(rot)
    wf_out.unpack(houtp[(e2e_steps - 1) % 2].cuda(), rot.shape, out=hres)
    torch.cuda.synchronize()
    e2e_packed_ok = bool(torch.equal(hres, drot[(e2e_steps - 1) % 2]))
    del hres, dinp, doutp
    del din, dprod, drot

    # ---- dominant kernel: the digit transforms (B x (L+1) rows of N = 2^14 per launch)
    ffi = eng.ffi
    ext = list(s.special_rings[0].prime_indices)
    ne = len(ext)
    buf = torch.empty((PAIRS, ne, N_DEG), dtype=torch.int64, device="cuda")
    for k, idx in enumerate(ext):
        buf[:, k].random_(0, s.special_rings[0].primes[k])
    limbs = ffi.new("uint32_t[]", ext)
    ptr = ffi.cast("uint64_t*", buf.data_ptr())
    sp = ffi.cast("void*", stream.cuda_stream)
    for _ in range(3):
        eng.lib.vfhe_cuda_ntt_batch(s.special_rings[0].NTT, 0, ptr, ptr, PAIRS, limbs, ne, sp)
    torch.cuda.synchronize()
    reps = 20
    profile_range(None, "digits", True)
    ev0.record(stream)
    for _ in range(reps):
        eng.lib.vfhe_cuda_ntt_batch(s.special_rings[0].NTT, 0, ptr, ptr, PAIRS, limbs, ne, sp)
    ev1.record(stream)
    torch.cuda.synchronize()
    profile_range(None, "digits", False)
    ntt_ms = ev0.elapsed_time(ev1) / reps
    sched = ffi.new("int32_t[3]")
    eng.lib.vfhe_cuda_ntt_get_schedule(14, PAIRS * ne, sched)
    kt = sched[0] or 12
    if kt >= 14:
        kname = f"k_tile_fwd_f<{kt},0>"
    elif sched[2] == -1:
        kname = f"k_fused_fwd_f<{kt},{14 - kt}> (thread-block cluster)"
    elif sched[2] == -2:
        kname = f"k_flow_f<{kt},{14 - kt}> (column and tile passes in one dataflow launch)"
    else:
        kname = f"k_col_f<{14 - kt},0> + k_tile_fwd_f<{kt},1>"
    alg_bytes = PAIRS * ne * 16 * N_DEG
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ntt_ms * 1e-3) / 1e9
    del buf

    # ---- secondary: N = 2^16, L = 24 forward NTT limbs/s (the NTT headline metric), on
    # 64 polynomials (805 MB, larger than L2, so every transform streams from HBM)
    from vfhe_b200.arith import Ring

    def ntt16_rate(split: int, profile: bool) -> tuple[float, float]:
        R16 = Ring(2**16, prime_size=[50] * 24, split_degree=split, engine=eng)
        b16 = torch.empty((NTT16_POLYS, 24, 2**16), dtype=torch.int64, device="cuda")
        for k, q in enumerate(R16.primes):
            b16[:, k].random_(0, q)
        l16 = ffi.new("uint32_t[]", R16.prime_indices)
        p16 = ffi.cast("uint64_t*", b16.data_ptr())
        for _ in range(3):
            eng.lib.vfhe_cuda_ntt_batch(R16.NTT, 0, p16, p16, NTT16_POLYS, l16, 24, sp)
        torch.cuda.synchronize()
        if profile:
            profile_range(None, "ntt16", True)
        ev0.record(stream)
        for _ in range(reps):
            eng.lib.vfhe_cuda_ntt_batch(R16.NTT, 0, p16, p16, NTT16_POLYS, l16, 24, sp)
        ev1.record(stream)
        torch.cuda.synchronize()
        if profile:
            profile_range(None, "ntt16", False)
        ms = ev0.elapsed_time(ev1) / reps
        del b16
        return ms, NTT16_POLYS * 24 / (ms * 1e-3)

    ms16, limbs16 = ntt16_rate(1, True)
    # the reference's default split for 50-bit primes: four 2^14-point blocks per limb
    ms16s4, limbs16s4 = ntt16_rate(4, False)
    eng.check("bench")
    # the reference's CPU figures (rank 0 at one GPU only): one core in this process and
    # all host cores in spawned processes
    pool = CpuPool() if (world == 1 and not args.no_cpu_baseline and _ref_library()[0].exists()) else None
    ntt16_cpu = {}
    if pool is not None:
        for split, tag in ((1, "split1"), (None, "split4")):
            one = _cpu_ntt_worker((16, 24, split, 3.0, SEED + 50))
            allc = pool.rate(_cpu_ntt_worker, (16, 24, split, 3.0), SEED + 51)
            ntt16_cpu[tag] = {"limbs_per_s_one_core": one["units"] / one["elapsed"],
                              "limbs_per_s_all_cores": allc["value"], "cores": allc["cores"], "kind": "reference",
                              "sample": f"polynomial_RNSc_to_RNS of one 24-limb polynomial, repeated for 3 s per "
                                        f"process, the reference's {one['engine']} engine"}
    encrypt = encrypt_leg(eng, s, key, d1[:, 1].contiguous(), reps=5)
    composed = composed_leg(eng) if world == 1 else None
    round_trip = ntt_round_trip_leg(eng, pool=pool)

    uneven = None if args.no_worklist else worklist_leg(eng, args.worklist_jobs, reps=max(3, min(args.steps, 10)),
                                                        cpu_budget=10.0 if pool is not None else 0.0)
    if pool is not None:
        pool.close()
    serving = None if args.no_serving else serving_leg(eng, args.serving_requests)
    cggi_fft = None if args.no_cggi else cggi_fft_leg(eng, 4096, reps=3, million=not args.no_cggi_million)
    rns_cggi = None if args.no_cggi else rns_cggi_leg(eng)

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- decoded error of one pair (host decode)
    from vfhe_b200.fhe import CKKS_Ciphertext
    from vfhe_b200.batch import to_host

    out_rows = to_host(rot[:1])[0]
    c = CKKS_Ciphertext(s, lvl=1)
    c.set_component_rows(0, out_rows[0])
    c.set_component_rows(1, out_rows[1])
    from vfhe_b200.arith import repr as prepr

    c.repr = prepr.coeff
    delta = SCALE * SCALE / s.rings[0].primes[-1]
    expect = np.roll(zs[0] * zs[1], -rot_steps[0])
    err = decoded_error(s, key, c, expect, delta)

    line = {
        "metric": "CKKS mul+relin+rescale/s",
        "value": value,
        "unit": "pairs/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": max(3, args.warmup),
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64 (RNS residues < 2^50)",
        "data": "synthetic (seeded keys, noise and unit-disk slots)",
        "config": dict(CONFIG, pairs_per_step=PAIRS, **({"ntt_schedule_override": args.ntt_schedule}
                                                         if args.ntt_schedule else {})),
        "e2e": {"value": e2e_value_plain, "unit": "pairs/s", "h2d_bytes_per_step": int(host1.nbytes + host2.nbytes),
                "d2h_bytes_per_step": int(hout[0].numel() * 8), "ms_per_step": e2e_ms_plain,
                "transport": "uint64 residue rows, the layout the cdef hands callers",
                "pipelining": "copy-in, compute and copy-out of consecutive steps overlap (two buffer sets)",
                "wire_format": {"value": e2e_value, "ms_per_step": e2e_ms,
                                "h2d_bytes_per_step": int(h1p.numel() + h2p.numel()),
                                "d2h_bytes_per_step": int(houtp[0].numel()),
                                "transport": "compact wire format (residues at their primes' bit lengths) as a "
                                             "client would send it: packed by the sender before the timed region, "
                                             "unpacked and packed on the GPU inside the step",
                                "packed_matches_plain": e2e_packed_ok},
                "wire_format_host_packed": {
                    "value": whole_job_rate(PAIRS, world, e2e_ms_hostpack), "ms_per_step": e2e_ms_hostpack,
                    "h2d_bytes_per_step": int(h1p.numel() + h2p.numel()),
                    "d2h_bytes_per_step": int(houtp[0].numel()), "host_threads": host_threads,
                    "transport": "compact wire format, packed from the uint64 rows and unpacked back into uint64 "
                                 "rows on the host inside the timed region (host wall clock)",
                    "unpacked_matches_device": hostpack_ok}},
        "roofline": {"bound": "hbm", "kernel": f"forward FP64 NTT, {kname} (digit transforms, {PAIRS * ne} rows x 2^14)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": MEASURED_TRAFFIC.get((kname, PAIRS * ne)), "launch_ms": ntt_ms,
                     "algorithmic_bytes": alg_bytes},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "decoded_max_error": err,
        "ntt_2p16_L24_split4": {"limbs_per_s": limbs16s4, "polys": NTT16_POLYS, "ms_per_launch": ms16s4,
                                "frac_hbm": 16 * 2**16 * limbs16s4 / 1e9 / peak,
                                **({"cpu_reference": ntt16_cpu["split4"]} if "split4" in ntt16_cpu else {})},
        "ntt_2p16_L24": {"limbs_per_s": limbs16, "polys": NTT16_POLYS, "ms_per_launch": ms16,
                         "frac_hbm": 16 * 2**16 * limbs16 / 1e9 / peak,
                         **({"cpu_reference": ntt16_cpu["split1"]} if "split1" in ntt16_cpu else {})},
    }
    if uneven is not None:
        line["uneven_worklist"] = uneven
    if serving is not None:
        line["serving"] = serving
    if cggi_fft is not None:
        line["cggi_fft_bootstrap"] = cggi_fft
    line["ckks_encrypt"] = encrypt
    if composed is not None:
        line["composed_ops"] = composed
    line["ntt_round_trip_n4096_L3"] = round_trip
    if rns_cggi is not None:
        line["cggi16_rns_bootstrap"] = rns_cggi
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--pairs", type=int, default=PAIRS,
                    help="ciphertext pairs per step (the workload is 256; smaller only for profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the reference CPU leg")
    ap.add_argument("--no-worklist", action="store_true", help="skip the uneven work-list leg")
    ap.add_argument("--worklist-jobs", type=int, default=512, help="jobs in the uneven work-list leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-loop leg")
    ap.add_argument("--no-cggi", action="store_true", help="skip the torus CGGI bootstrap leg")
    ap.add_argument("--no-cggi-million", action="store_true",
                    help="skip bootstrapping 10^6 LWEs to count lookup mismatches (about a minute)")
    ap.add_argument("--serving-requests", type=int, default=200, help="requests per arrival rate in the serving leg")
    ap.add_argument("--ntt-schedule", action="append", default=[], metavar="LOGP:K,TPC,CPS",
                    help="override the tuned transform schedule of every row-count class of 2^LOGP-point rows "
                         "(vfhe_cuda_ntt_set_schedule), e.g. 14:10,2,-2 for the dataflow launch")
    ap.add_argument("--profile-leg", default="ckks", choices=["ckks", "digits", "ntt16", "cggi_fft", "cggi_rns", "worklist", "worklist_graph",
                             "roundtrip", "roundtrip_split1", "encrypt"],
                    help="leg whose timed region is the profiler capture range (ncu --profile-from-start off)")
    args = ap.parse_args()
    global PROFILE_LEG
    PROFILE_LEG = args.profile_leg
    sys.path.insert(0, str(ROOT))
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        run_reference_arm(args)
    else:
        run_cuda_arm(args)


if __name__ == "__main__":
    main()
