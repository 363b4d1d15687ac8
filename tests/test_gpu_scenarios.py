"""cuda engine vs the CPU oracle on whole pipelines (§8 rows a8-a15), bit for bit.

Inputs are seeded and identical on both engines (tests/scenarios.py), so any
difference in a residue is an engine difference.
"""

from __future__ import annotations

import numpy as np
import pytest

from . import scenarios
from .test_scenarios_oracle import compare

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["keyswitch", "multiply", "automorphism", "cmux"])
def test_pipeline_parity(name, cuda, oracle_engine):
    fn = getattr(scenarios, name)
    compare(fn(cuda), fn(oracle_engine))


def test_automorphism_split4(cuda, oracle_engine):
    compare(scenarios.automorphism(cuda, split=4), scenarios.automorphism(oracle_engine, split=4))


def test_keyswitch_two_special_primes(cuda, oracle_engine):
    compare(scenarios.keyswitch(cuda, L=3, special=2), scenarios.keyswitch(oracle_engine, L=3, special=2))


def test_ckks_small(cuda, oracle_engine):
    a = scenarios.ckks_pipeline(cuda)
    b = scenarios.ckks_pipeline(oracle_engine)
    compare(a, b)
    assert a["mul_err"] < 1e-6 and a["rot1_err"] < 1e-6 and a["rot3_err"] < 1e-6


def test_ckks_config_shape(cuda, oracle_engine):
    """N = 2^14, one 50-bit base prime, eight 40-bit primes, one 50-bit special prime,
    scale 2^40: multiply -> relinearise -> rescale -> rotate by 2^3."""
    a = scenarios.ckks_pipeline(cuda, N=2**14, n_mid=8, steps=(8,))
    b = scenarios.ckks_pipeline(oracle_engine, N=2**14, n_mid=8, steps=(8,))
    compare(a, b)
    # decoded max error vs the FP64 plaintext: ~1.8e-8 after mul+rescale (the reference
    # measures the same), ~1.4e-6 after the rotation's key switch
    assert a["mul_err"] < 1e-6 and a["rot8_err"] < 1e-4, (a["mul_err"], a["rot8_err"])


def test_cggi_bootstrap(cuda, oracle_engine):
    a = scenarios.cggi_bootstrap(cuda)
    b = scenarios.cggi_bootstrap(oracle_engine)
    compare(a, b)
    assert all(a["ok"])


def test_cggi_bootstrap_n1024(cuda, oracle_engine):
    """Reference comparison point for the CGGI configuration: ring N = 1024 with three
    50-bit primes (one special), RNS gadget, LWE dimension 64 (bounded for the oracle)."""
    a = scenarios.cggi_bootstrap(cuda, N=1024, n_lwe=64, count=2)
    b = scenarios.cggi_bootstrap(oracle_engine, N=1024, n_lwe=64, count=2)
    compare(a, b)
    assert all(a["ok"])


def test_full_packing_keyswitch_matches_reference_library(cuda, ref_portable):
    """mlwe_full_packing_keyswitch (mlwe.c:343-430, GP25's LWE repacking): the same
    samples and packing key on the cuda engine and on the reference's own library
    give the same MLWE, residue for residue."""
    from tests.helpers import twin_rings
    from vfhe_b200.arith import repr
    from vfhe_b200.mlwe import LWE, MLWE, MLWE_Scheme, MLWE_Set

    N, size = 256, 8
    rng = np.random.default_rng(41)
    outs = []
    rings = twin_rings([cuda, ref_portable], N, [50, 50, 50], split=1)
    rows_lwe = [(np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in rings[0].primes[:2]]),
                 [int(rng.integers(0, q)) for q in rings[0].primes[:2]]) for _ in range(size)]
    key_rows = [[np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in rings[0].primes])
                           for _ in range(2)]) for _ in range(2)] for _ in range(N)]
    for R in rings:
        s = MLWE_Scheme(R, special_primes=1, module_rank=1, max_lvl=1)
        lwes = []
        for a, b in rows_lwe:
            c = LWE(s.rings[0], n=N)
            c.set_rows(a, b)
            lwes.append(c)
        comps = []
        for i in range(N):
            row = []
            for d in range(2):
                k = MLWE(s, ring=s.special_rings[0])
                k.set_component_rows(0, key_rows[i][d][0])
                k.set_component_rows(1, key_rows[i][d][1])
                k.repr = repr.ntt
                row.append(k)
            comps.append(row)
        ksk = MLWE_Set(comps)
        res = MLWE(s, lvl=0)
        arr = R.ffi.new("void*[]", [c.obj for c in lwes])
        R.lib.mlwe_full_packing_keyswitch(res.obj, arr, size, ksk.obj, 0)
        R.engine.check("mlwe_full_packing_keyswitch")
        outs.append(np.stack([res.component_rows(0), res.component_rows(1)]))
    assert np.array_equal(outs[0], outs[1])


def test_trace_matches_reference_library(cuda, ref_portable):
    """mlwe_trace (mlwe.c:436-444 over mlwe_partial_trace, mlwe.c:328-341: log2 N automorphism key
    switches and additions) on the cuda engine and on the reference's own library,
    with the same (random) key material: the same MLWE, residue for residue."""
    from tests.helpers import twin_rings
    from vfhe_b200.arith import repr
    from vfhe_b200.mlwe import MLWE, MLWE_Scheme, MLWE_Set

    N = 256
    logN = 8
    rng = np.random.default_rng(43)
    rings = twin_rings([cuda, ref_portable], N, [50, 50, 50], split=1)
    ct_rows = [np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in rings[0].primes[:2]]) for _ in range(2)]
    key_rows = [[np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in rings[0].primes])
                           for _ in range(2)]) for _ in range(2)] for _ in range(logN)]
    outs = []
    for R in rings:
        s = MLWE_Scheme(R, special_primes=1, module_rank=1, max_lvl=1)
        c = MLWE(s, lvl=0)
        c.set_component_rows(0, ct_rows[0])
        c.set_component_rows(1, ct_rows[1])
        c.repr = repr.coeff
        sets = []
        for g in range(logN):
            digits = []
            for d in range(2):
                k = MLWE(s, ring=s.special_rings[0])
                k.set_component_rows(0, key_rows[g][d][0])
                k.set_component_rows(1, key_rows[g][d][1])
                k.repr = repr.ntt
                digits.append(k)
            sets.append(MLWE_Set([digits]))
        ksks = MLWE_Set.flatten_array(sets)
        out = MLWE(s, lvl=0)
        R.lib.mlwe_trace(out.obj, c.obj, ksks.obj, 0)
        R.engine.check("mlwe_trace")
        outs.append(np.stack([out.component_rows(0), out.component_rows(1)]))
    assert np.array_equal(outs[0], outs[1])


def _mlwe_rows(rng, primes, N, count):
    return [np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in primes]) for _ in range(2)])
            for _ in range(count)]


def _mlwe_array(s, ring, rows, rep):
    """An engine-side RNS_MLWE* array (MGSW layout) from [2][limbs][N] row sets."""
    from vfhe_b200.mlwe import MLWE

    objs = []
    for r in rows:
        m = MLWE(s, ring=ring)
        m.set_component_rows(0, r[0])
        m.set_component_rows(1, r[1])
        m.repr = rep
        objs.append(m)
    tmp = ring.ffi.new("void*[]", [m.obj for m in objs])
    arr = ring.lib.mlwe_create_copy_array(tmp, len(objs))
    return arr, objs


def test_gp25_steps_match_reference_library(cuda, ref_portable):
    """GP25's C steps (gp25.c:68-336): the RGSW monomial multiply (NCMUX/CMUX rounds
    over the accumulators) and sub_a (rotate, external product with the sign key,
    add) on the cuda engine and on the reference's own library, same inputs: the same
    accumulators, residue for residue."""
    from tests.helpers import twin_rings
    from vfhe_b200.arith import repr
    from vfhe_b200.mlwe import MLWE, MLWE_Scheme, MLWE_Set

    N, in_N, r_prec, ell = 256, 4, 2, 2
    rng = np.random.default_rng(47)
    rings = twin_rings([cuda, ref_portable], N, [50, 50, 50], split=1)
    primes = rings[0].primes
    acc_rows = _mlwe_rows(rng, primes[:2], N, in_N)
    e_rows = [_mlwe_rows(rng, primes, N, 2 * ell) for _ in range(r_prec)]
    k_rows = _mlwe_rows(rng, primes, N, ell)
    sign_rows = _mlwe_rows(rng, primes, N, 2 * ell)
    rots = [int(v) for v in rng.integers(0, 2 * N, in_N)]
    results = []
    for R in rings:
        s = MLWE_Scheme(R, special_primes=1, module_rank=1, max_lvl=1)
        sr = s.special_rings[0]
        outs = []
        for step in ("monomial", "sub_a"):
            accs = []
            for rows in acc_rows:
                m = MLWE(s, lvl=0)
                m.set_component_rows(0, rows[0])
                m.set_component_rows(1, rows[1])
                m.repr = repr.coeff
                accs.append(m)
            p0 = R.ffi.new("void*[]", [m.obj for m in accs])
            keep = []
            if step == "monomial":
                es = [_mlwe_array(s, sr, rows, repr.ntt) for rows in e_rows]
                keep += es
                e = R.ffi.new("void*[]", [a for a, _ in es])
                digits = []
                for rows in k_rows:
                    k = MLWE(s, ring=sr)
                    k.set_component_rows(0, rows[0])
                    k.set_component_rows(1, rows[1])
                    k.repr = repr.ntt
                    digits.append(k)
                ksk = MLWE_Set([digits])
                keep.append(ksk)
                R.lib.gp25_RGSW_monomial_mul(p0, in_N, e, r_prec, ksk.obj, ell, 1)
                R.engine.check("gp25_RGSW_monomial_mul")
            else:
                sign, objs = _mlwe_array(s, sr, sign_rows, repr.ntt)
                keep.append(objs)
                R.lib.gp25_sub_a_mt(p0, in_N, R.ffi.new("uint64_t[]", rots), sign, ell, 1, N, 1)
                R.engine.check("gp25_sub_a_mt")
            outs.append(np.stack([np.stack([m.component_rows(0), m.component_rows(1)]) for m in accs]))
        results.append(outs)
    for got, want in zip(results[0], results[1]):
        assert np.array_equal(got, want)
