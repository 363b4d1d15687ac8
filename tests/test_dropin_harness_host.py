"""Host checks of the drop-in harness (no GPU).

* The reference's engine picker (modules/misc/python/src/_vfhe_native.py:29-56) selects
  the cffi module `_vfhe_native_cuda` built against include/vfhe_cuda.h when
  VFHE_ENGINE=cuda, and that module links the engine library (import only: no GPU call).
* The child-process driver used by the GPU orchestration tests reproduces a result on
  the reference's two engines from injected inputs: dump on one engine, inject into the
  other, identical outputs (the reference's engines agree bit for bit on these paths).
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import build_dropin  # noqa: E402

BUILT = (build_dropin.BUILD / "_vfhe_engines.py").exists()
pytestmark = pytest.mark.skipif(not BUILT, reason="drop-in harness not built (python oracle/build_dropin.py)")


def _env(engine: str) -> dict:
    return dict(os.environ, VFHE_ENGINE=engine, PYTHONPATH=build_dropin.pythonpath(), PYTHONDONTWRITEBYTECODE="1")


def test_picker_loads_cuda_module_without_gpu():
    code = "import _vfhe_native as n; print(n.active, n.ffi.string(n.lib.vfhe_engine_active()).decode())"
    r = subprocess.run([sys.executable, "-c", code], env=_env("cuda"), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.split() == ["cuda", "cuda"]


def test_driver_injection_reproduces_across_reference_engines(tmp_path):
    engines = build_dropin.BUILD.joinpath("_vfhe_engines.py").read_text()
    if "avx512ifma" not in engines or "avx512ifma" not in Path("/proc/cpuinfo").read_text():
        pytest.skip("needs both reference engines")
    for engine, mode in (("avx512ifma", "make"), ("portable", "inject")):
        r = subprocess.run([sys.executable, "-W", "ignore", str(ROOT / "tests" / "dropin_driver.py"), "ckks", mode,
                            str(tmp_path)], env=_env(engine), capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stdout + r.stderr
    a, b = np.load(tmp_path / "out_avx512ifma.npz"), np.load(tmp_path / "out_portable.npz")
    for k in a:
        assert np.array_equal(a[k], b[k]), k
