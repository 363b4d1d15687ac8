"""mlwe_full_packing_keyswitch's batched inner product (every mask entry's digits built,
transformed and multiplied into the packing key in a few launches per chunk) against
the sequential form (one digit polynomial per mask entry), at N = 2048 with LWE
dimension 2048: 4096 digits in three chunks, so the chunks' partial sums are added.
The sequential form is checked against the reference's own library at N = 256
(test_gpu_scenarios.py)."""

from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batched_packing_matches_sequential(cuda):
    from vfhe_b200.arith import Ring, repr
    from vfhe_b200.mlwe import LWE, MLWE, MLWE_Scheme, MLWE_Set

    N, size = 2048, 24
    rng = np.random.default_rng(71)
    R = Ring(N, prime_size=[50, 50, 50], split_degree=1, engine=cuda)
    s = MLWE_Scheme(R, special_primes=1, module_rank=1, max_lvl=1)
    lwes = []
    for _ in range(size):
        x = LWE(s.rings[0], n=N)
        x.set_rows(np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in R.primes[:2]]),
                   [int(rng.integers(0, q)) for q in R.primes[:2]])
        lwes.append(x)
    comps = []
    for _ in range(N):
        row = []
        for _ in range(2):
            k = MLWE(s, ring=s.special_rings[0])
            k.set_component_rows(0, np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in R.primes]))
            k.set_component_rows(1, np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in R.primes]))
            k.repr = repr.ntt
            row.append(k)
        comps.append(row)
    ksk = MLWE_Set(comps)
    arr = R.ffi.new("void*[]", [x.obj for x in lwes])
    outs = []
    old = os.environ.get("VFHE_CUDA_PACKING_SEQUENTIAL")
    try:
        for sequential in ("0", "1"):
            os.environ["VFHE_CUDA_PACKING_SEQUENTIAL"] = sequential
            res = MLWE(s, lvl=0)
            R.lib.mlwe_full_packing_keyswitch(res.obj, arr, size, ksk.obj, 0)
            cuda.check("mlwe_full_packing_keyswitch")
            outs.append(np.stack([res.component_rows(0), res.component_rows(1)]))
    finally:
        if old is None:
            os.environ.pop("VFHE_CUDA_PACKING_SEQUENTIAL", None)
        else:
            os.environ["VFHE_CUDA_PACKING_SEQUENTIAL"] = old
    assert np.array_equal(outs[0], outs[1])
    assert outs[0].any()
