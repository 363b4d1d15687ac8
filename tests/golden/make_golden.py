"""Generate the golden fixtures in this folder from the reference's own C library.

Run from the repository root after oracle/build_ref.sh has built the reference's
portable engine from its sources (oracle/_ref/libvfhe_ref_portable.so):

    python tests/golden/make_golden.py

Writes ntt_kats.json:
  * "forward": for the rings of the independent known-answer table in
    tests/test_golden.py (N=4096 at split 4 and 1, and the N=2^14 CKKS chain) -- limb-0 input (0x123456789ABCDEF + i) mod q in the
    raw row layout, forward transform through polynomial_RNSc_to_RNS; the ring primes,
    the first 64 outputs of every limb, a SHA-256 of all output rows, and w[0][0:8] of
    the pool's twist table;
  * "negacyclic": the convolution theorem case of the reference's test_ntt.c
    (a[i] = (i + 123) mod q, b[i] = (2 i + 456) mod q, q = the first prime above 2^bits
    with q = 2n + 1 mod 4n) as polynomial_RNSc_to_RNS, polynomial_mul_RNS_polynomial,
    polynomial_RNS_to_RNSc at split 1; the product is also computed by schoolbook here
    and must agree before anything is written.
"""

from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

FORWARD_RINGS = [
    {"N": 4096, "prime_size": [50, 50, 50], "split": None},
    {"N": 4096, "prime_size": [50, 50, 50], "split": 1},
    {"N": 2**14, "prime_size": [50] + [40] * 8 + [50], "split": 1},
]
NEGACYCLIC = [(n, bits) for n in (64, 256, 1024) for bits in (20, 40, 50)]


def special_prime_above(x: int, n: int) -> int:
    """First prime q > x with q = 1 mod 2n and q != 1 mod 4n (number_theory.c:179-210)."""
    from vfhe_b200.numbers import is_prime

    order = 2 * n
    a = x // order
    if a * order + 1 <= x:
        a += 1
    if a % 2 == 0:
        a += 1
    while not is_prime(a * order + 1):
        a += 2
    return a * order + 1


def schoolbook(a: list[int], b: list[int], q: int) -> list[int]:
    n = len(a)
    out = [0] * n
    for i in range(n):
        for j in range(n):
            p = a[i] * b[j]
            if i + j < n:
                out[i + j] += p
            else:
                out[i + j - n] -= p
    return [v % q for v in out]


def digest(rows: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(rows, dtype=np.uint64).tobytes()).hexdigest()


def forward_case(engine, spec: dict) -> dict:
    from vfhe_b200.arith import Polynomial, Ring, repr, reset_registries

    reset_registries()
    R = Ring(spec["N"], prime_size=spec["prime_size"], split_degree=spec["split"], engine=engine)
    rows = np.stack([(0x123456789ABCDEF + np.arange(R.N, dtype=object)) % q for q in R.primes]).astype(np.uint64)
    p = Polynomial(R)
    p.set_rows(rows)
    p.rns_mask = R.mask
    p.repr = repr.coeff
    p.to_NTT()
    out = p.rows()
    w = engine.ffi.cast("incNTT", R.NTT).w
    w0 = [int(w[R.prime_indices[0]][i]) for i in range(8)]
    return {"N": R.N, "prime_size": spec["prime_size"], "split": R.split_degree, "primes": R.primes,
            "head": [[int(v) for v in out[k, :64]] for k in range(len(R.primes))], "sha256": digest(out),
            "w0": w0}


def negacyclic_case(engine, n: int, bits: int) -> dict:
    from vfhe_b200.arith import Polynomial, Ring, repr, reset_registries

    reset_registries()
    q = special_prime_above(1 << bits, n)
    R = Ring(n, primes=[q], prime_size=[bits + 1], split_degree=1, engine=engine)
    a = [(i + 123) % q for i in range(n)]
    b = [(2 * i + 456) % q for i in range(n)]
    want = schoolbook(a, b, q)
    pa, pb = Polynomial(R), Polynomial(R)
    for p, v in ((pa, a), (pb, b)):
        p.set_rows(np.array([v], dtype=np.uint64))
        p.rns_mask = R.mask
        p.repr = repr.coeff
    c = pa * pb
    c.to_coeff()
    got = [int(v) for v in c.rows()[0]]
    assert got == want, (n, bits)
    return {"n": n, "bits": bits, "q": q, "head": want[:32], "sha256": digest(np.array([want], dtype=np.uint64))}


def main() -> None:
    from vfhe_b200.native import Engine

    lib = ROOT / "oracle" / "_ref" / "libvfhe_ref_portable.so"
    if not lib.exists():
        raise SystemExit("build the reference library first: oracle/build_ref.sh")
    eng = Engine(lib)
    out = {"generator": "tests/golden/make_golden.py on the reference's portable engine (oracle/_ref)",
           "forward": [forward_case(eng, s) for s in FORWARD_RINGS],
           "negacyclic": [negacyclic_case(eng, n, b) for n, b in NEGACYCLIC]}
    (Path(__file__).parent / "ntt_kats.json").write_text(json.dumps(out, indent=1))
    print("wrote", Path(__file__).parent / "ntt_kats.json")


if __name__ == "__main__":
    main()
