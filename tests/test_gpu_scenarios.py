"""cuda engine vs the CPU oracle on whole pipelines (§8 rows a8-a15), bit for bit.

Inputs are seeded and identical on both engines (tests/scenarios.py), so any
difference in a residue is an engine difference.
"""

from __future__ import annotations

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
