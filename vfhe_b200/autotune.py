"""Autotuner for the transform launch schedule (vfhe_cuda_ntt_set_schedule).

For a (log2 P, rows-per-launch) class the tuner times every candidate schedule of the
FP64 transform -- tile bits (one pass, or a radix-2^(logP - tile_bits) column pass
followed by tiles), tiles per CTA, and one-CTA-per-tile-group vs a persistent grid of
k CTAs per SM -- on forward + inverse transforms of that many rows, and keeps the
fastest.  Schedules never change results (the transform is exact), so a tuned table
can be applied at any time.  The table is a JSON file keyed "logP/rows_log2";
``apply`` loads it into the engine and missing classes use the nearest tuned bucket
of the same logP.

    python -m vfhe_b200.autotune --out vfhe_b200/tuned/ntt_schedule_b200.json
"""

from __future__ import annotations

import argparse
import json
from pathlib import Path

import numpy as np

from .native import Engine, cuda_engine

DEFAULT_TABLE = Path(__file__).resolve().parent / "tuned" / "ntt_schedule_b200.json"
MAX_ELEMS = 1 << 28  # at most 2 GiB of rows per timed buffer
BUCKETS = (4, 7, 9, 11, 13, 15)
KEEP_DEFAULT_MARGIN = 0.03  # a tuned schedule must beat the built-in one by 3%


def candidates(logP: int) -> list[tuple[int, int, int]]:
    """(tile_bits, tiles_per_cta, ctas_per_sm) triples worth timing for one logP."""
    if logP <= 13:  # one pass, or a short column pass in front of smaller tiles
        tiles = {k for k in (logP, logP - 1, logP - 2) if k >= 8}
    else:  # a column pass of radix 2^(logP - k) is required
        tiles = set(range(max(8, logP - 5), 14))
    out = []
    for k in sorted(tiles):
        tpt = 1 << (k - 4)
        tpcs = [0] + [t for t in (1, 2, 4, 8) if tpt * t <= max(256, tpt) and tpt * t >= 64]
        for tpc in sorted(set(tpcs)):
            for cps in (0, 2, 4):
                out.append((k, tpc, cps))
    # fused split transforms on a thread-block cluster of 2^(logP - k) CTAs (ctas_per_sm = -1)
    for k in (11, 12, 13):
        if 1 <= logP - k <= 3:
            out.append((k, 0, -1))
    # column pass and tile pass as one dataflow launch (ctas_per_sm = -2; tiles_per_cta =
    # work items per ticket)
    for k in (10, 11, 12, 13):
        if flow_supported(k, logP - k):
            out.extend((k, per, -2) for per in (1, 2))
    return out


def flow_supported(k: int, k1: int) -> bool:
    """Shapes of the dataflow launch (ntt_flow.cu): 2^k-point tiles, a radix-2^k1 column
    pass, and the tiles of one 256-thread item in one row."""
    if not (10 <= k <= 13 and 2 <= k1 <= 4):
        return False
    per_item = 1 if k >= 12 else (2 if k == 11 else 4)
    return per_item <= (1 << k1)


def _time_shape(engine: Engine, logP: int, rows: int, cands, reps: int = 5) -> list[tuple[float, tuple]]:
    import torch

    from .arith import Ring

    ffi, lib = engine.ffi, engine.lib
    N = 1 << logP
    L = 4
    R = Ring(N, prime_size=[50] * L, split_degree=1, engine=engine)
    batch = max(1, rows // L)
    buf = torch.empty((batch, L, N), dtype=torch.int64, device="cuda")
    for k, q in enumerate(R.primes):
        buf[:, k].random_(0, q)
    limbs = ffi.new("uint32_t[]", R.prime_indices)
    p = ffi.cast("uint64_t*", buf.data_ptr())
    st = torch.cuda.current_stream()
    sp = ffi.cast("void*", st.cuda_stream)
    bucket = (batch * L).bit_length() - 1
    res = []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for c in cands:
        if lib.vfhe_cuda_ntt_set_schedule(logP, bucket, *c) != 0:
            lib.vfhe_cuda_clear_error()
            continue
        for _ in range(2):
            lib.vfhe_cuda_ntt_batch(R.NTT, 0, p, p, batch, limbs, L, sp)
            lib.vfhe_cuda_ntt_batch(R.NTT, 1, p, p, batch, limbs, L, sp)
        ev0.record(st)
        for _ in range(reps):
            lib.vfhe_cuda_ntt_batch(R.NTT, 0, p, p, batch, limbs, L, sp)
            lib.vfhe_cuda_ntt_batch(R.NTT, 1, p, p, batch, limbs, L, sp)
        ev1.record(st)
        torch.cuda.synchronize()
        res.append((ev0.elapsed_time(ev1) / reps, c))
    lib.vfhe_cuda_ntt_set_schedule(logP, bucket, 0, 0, 0)
    engine.check("autotune")
    return sorted(res)


def tune(engine: Engine | None = None, logps=range(8, 18), buckets=BUCKETS, reps: int = 5,
         verbose: bool = False) -> dict:
    """Time every candidate for each (logP, bucket) that fits MAX_ELEMS; returns the table."""
    engine = engine or cuda_engine()
    table = {}
    for logP in logps:
        cands = candidates(logP)
        for b in buckets:
            rows = 1 << b
            if rows << logP > MAX_ELEMS or rows < 4:
                continue
            timed = _time_shape(engine, logP, rows, cands, reps)
            if not timed:
                continue
            best_ms, best = timed[0]
            default_ms = next((ms for ms, c in timed if c == (logP if logP <= 13 else 12, 0, 0)), None)
            if default_ms is not None and best_ms > (1.0 - KEEP_DEFAULT_MARGIN) * default_ms:
                best_ms, best = default_ms, (logP if logP <= 13 else 12, 0, 0)  # not worth a change
            table[f"{logP}/{b}"] = {"schedule": list(best), "ms": best_ms, "default_ms": default_ms}
            if verbose:
                print(f"logP={logP} rows=2^{b}: best {best} {best_ms:.3f} ms (default {default_ms})", flush=True)
    return table


def apply(engine: Engine, table: dict) -> int:
    """Load a tuned table into the engine; every bucket of a tuned logP gets the nearest
    tuned entry.  Returns the number of (logP, bucket) classes set."""
    by_logp: dict[int, dict[int, list[int]]] = {}
    for key, val in table.items():
        lp, b = (int(x) for x in key.split("/"))
        by_logp.setdefault(lp, {})[b] = val["schedule"]
    n = 0
    for lp, entries in by_logp.items():
        tuned = sorted(entries)
        for b in range(32):
            near = min(tuned, key=lambda t: (abs(t - b), t))
            if engine.lib.vfhe_cuda_ntt_set_schedule(lp, b, *entries[near]) != 0:
                engine.lib.vfhe_cuda_clear_error()
                continue
            n += 1
    return n


def load(path: Path = DEFAULT_TABLE) -> dict | None:
    try:
        return json.loads(Path(path).read_text())["table"]
    except (OSError, ValueError, KeyError):
        return None


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(DEFAULT_TABLE))
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--logp", type=int, nargs="*", default=None, help="tune only these log2 P (default 8..17)")
    ap.add_argument("--merge", action="store_true", help="keep the --out table's entries for other log2 P")
    args = ap.parse_args()
    import torch

    eng = cuda_engine(apply_tuned=False)
    table = tune(eng, logps=args.logp or range(8, 18), reps=args.reps, verbose=True)
    if args.merge:
        old = load(Path(args.out)) or {}
        old.update(table)
        table = old
    out = {"device": torch.cuda.get_device_name(0), "table": table,
           "note": "ms = forward + inverse transform of 2^bucket rows of 2^logP, CUDA events"}
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    Path(args.out).write_text(json.dumps(out, indent=1, sort_keys=True))
    gains = [v["default_ms"] / v["ms"] for v in table.values() if v.get("default_ms")]
    print(f"tuned {len(table)} classes; median gain over default {np.median(gains):.3f}x, max {max(gains):.3f}x")


if __name__ == "__main__":
    main()
