"""Pins the CPU oracle's mlwe/fhe pipelines to the reference library: each scenario
runs on the oracle and on the reference built from its own sources, bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from . import scenarios


def compare(a: dict, b: dict) -> None:
    for key, va in a.items():
        vb = b[key]
        if isinstance(va, np.ndarray):
            assert va.shape == vb.shape, key
            assert np.array_equal(va, vb), f"{key}: {(va != vb).sum()} residues differ"
        elif isinstance(va, list) and va and isinstance(va[0], np.ndarray):
            for x, y in zip(va, vb):
                assert np.array_equal(x, y), key
        elif isinstance(va, float) and key.endswith("err"):
            continue  # decode errors are checked by the callers
        else:
            assert va == vb, key


@pytest.mark.parametrize("name", ["keyswitch", "multiply", "automorphism", "cmux"])
def test_oracle_matches_reference(name, oracle_engine, ref_portable):
    fn = getattr(scenarios, name)
    compare(fn(oracle_engine), fn(ref_portable))


def test_oracle_ckks_pipeline(oracle_engine, ref_portable):
    a = scenarios.ckks_pipeline(oracle_engine)
    b = scenarios.ckks_pipeline(ref_portable)
    compare(a, b)
    assert a["mul_err"] < 1e-6 and a["rot1_err"] < 1e-6, a


def test_oracle_cggi_bootstrap(oracle_engine, ref_portable):
    a = scenarios.cggi_bootstrap(oracle_engine, n_lwe=8, count=1)
    b = scenarios.cggi_bootstrap(ref_portable, n_lwe=8, count=1)
    compare(a, b)
    assert all(a["ok"])
