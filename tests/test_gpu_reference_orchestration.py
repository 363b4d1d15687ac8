"""The reference's own CKKS and CGGI16 orchestration, residue for residue, on the cuda engine.

`tests/dropin_driver.py` runs the reference's classes (CKKS_Ciphertext.__mul__ and
CKKS_Scheme.rotate, modules/fhe/python/src/vfhe/fhe/ckks.py:110-119,227-241;
CGGI16.functional_bootstrap, modules/fhe/python/src/vfhe/fhe/cggi16.py:115-128) in child
processes: once on the reference's own engine, which draws the keys and ciphertexts and
dumps them, and once with VFHE_ENGINE=cuda on those injected inputs.  The outputs must be
identical.  Shapes: the CKKS configuration (N = 2^14, [50] + [40]*8 + [50], one special
prime), and the CGGI16 bootstrap at N = 1024 with an LWE dimension of 630.
"""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from .conftest import has_ifma

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import build_dropin  # noqa: E402


def run_driver(scenario: str, mode: str, engine: str, d: Path) -> None:
    env = dict(os.environ, VFHE_ENGINE=engine, PYTHONPATH=build_dropin.pythonpath(), PYTHONDONTWRITEBYTECODE="1")
    env.pop("VFHE_CUDA_QUIET", None)
    r = subprocess.run([sys.executable, "-W", "ignore", str(ROOT / "tests" / "dropin_driver.py"), scenario, mode,
                        str(d)], env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout + r.stderr


def reference_engine(scenario: str) -> str:
    built = (build_dropin.BUILD / "_vfhe_engines.py").read_text()
    # the IFMA engine skips the n mod 8 tail of LWE operations (mod50.c:93), so the
    # n = 630 LWE inputs of the CGGI scenario come from the portable engine
    if scenario == "ckks" and has_ifma() and "avx512ifma" in built:
        return "avx512ifma"
    return "portable"


@pytest.mark.parametrize("scenario", ["ckks", "cggi"])
def test_reference_orchestration_matches_on_cuda(scenario, tmp_path):
    if not (build_dropin.BUILD / "_vfhe_engines.py").exists():
        pytest.fail(f"{build_dropin.OUT} is not built: run `python oracle/build_dropin.py`")
    ref = reference_engine(scenario)
    run_driver(scenario, "make", ref, tmp_path)
    run_driver(scenario, "inject", "cuda", tmp_path)
    want, got = np.load(tmp_path / f"out_{ref}.npz"), np.load(tmp_path / "out_cuda.npz")
    for k in want:
        assert want[k].shape == got[k].shape, k
        bad = np.argwhere(want[k] != got[k])
        assert bad.size == 0, f"{k}: {len(bad)} residues differ, first at {bad[0].tolist()}"
    info = json.loads((tmp_path / f"info_{ref}.json").read_text())
    if scenario == "ckks":
        assert info["decoded_max_error"] < 1e-4
    else:
        assert info["decrypted"] == info["expected"]
        assert json.loads((tmp_path / "info_cuda.json").read_text())["decrypted"] == info["expected"]
