"""Shared fixtures.

``gpu`` marks tests that need a CUDA device (the cuda engine has no CPU path).
The CPU oracle (oracle/vfhe_oracle.c, built to oracle/_build/) is loaded only here,
as the checker; the reference libraries under oracle/_ref/ are used when present.
"""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
ORACLE_SRC = ROOT / "oracle" / "vfhe_oracle.c"
ORACLE_LIB = ROOT / "oracle" / "_build" / "libvfhe_oracle.so"
REF_DIR = ROOT / "oracle" / "_ref"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built cuda engine")


def build_oracle() -> Path:
    """Compile the C oracle if its library is missing or stale."""
    if not ORACLE_LIB.exists() or ORACLE_LIB.stat().st_mtime < ORACLE_SRC.stat().st_mtime:
        ORACLE_LIB.parent.mkdir(exist_ok=True)
        subprocess.run(
            ["gcc", "-O2", "-std=gnu11", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(ORACLE_LIB), str(ORACLE_SRC), "-lm"],
            check=True,
        )
    return ORACLE_LIB


TORUS_SRC = ROOT / "oracle" / "cggi_torus_oracle.c"
TORUS_LIB = ROOT / "oracle" / "_build" / "libcggi_torus_oracle.so"


def build_torus_oracle() -> Path:
    """Compile the exact-integer torus CGGI oracle if missing or stale."""
    if not TORUS_LIB.exists() or TORUS_LIB.stat().st_mtime < TORUS_SRC.stat().st_mtime:
        TORUS_LIB.parent.mkdir(exist_ok=True)
        subprocess.run(["gcc", "-O3", "-std=gnu11", "-fPIC", "-shared", "-o", str(TORUS_LIB), str(TORUS_SRC)],
                       check=True)
    return TORUS_LIB


@pytest.fixture(scope="session")
def torus_oracle():
    """ctypes handle on the exact torus CGGI oracle (checker only)."""
    import ctypes

    lib = ctypes.CDLL(str(build_torus_oracle()))
    u32p, i32p = ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_int32)
    lib.tor_external_product.argtypes = [u32p, u32p, u32p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.tor_bootstrap.argtypes = [u32p, u32p, ctypes.c_uint32, u32p, u32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_uint32]
    lib.tor_keyswitch.argtypes = [u32p, u32p, u32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.tor_negacyclic_mac.argtypes = [u32p, i32p, u32p, ctypes.c_int]
    lib.tor_decompose.argtypes = [i32p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int]
    return lib


@pytest.fixture(scope="session")
def oracle_engine():
    from vfhe_b200.native import Engine

    return Engine(build_oracle(), "oracle")


def ref_engine_path(name: str) -> Path | None:
    p = REF_DIR / f"libvfhe_ref_{name}.so"
    return p if p.exists() else None


@pytest.fixture(scope="session")
def ref_portable():
    from vfhe_b200.native import Engine

    p = ref_engine_path("portable")
    if p is None:
        pytest.skip("reference library not built (oracle/build_ref.sh)")
    return Engine(p)


@pytest.fixture(scope="session")
def cuda():
    from vfhe_b200.native import cuda_engine

    return cuda_engine()


@pytest.fixture(autouse=True)
def _fresh_prime_pools():
    """Each test starts with empty prime pools, as in the reference's conftest.py:63-85."""
    from vfhe_b200.arith import reset_registries

    reset_registries()
    yield
    reset_registries()


@pytest.fixture(autouse=True)
def _no_device_faults(request):
    """After every GPU test: no kernel's bounded wait for a bulk copy gave up (a wait
    that gives up raises a device flag and leaves wrong results behind)."""
    yield
    if request.node.get_closest_marker("gpu") is None:
        return
    from vfhe_b200 import native

    eng = native._CUDA
    if eng is None:
        return
    assert eng.lib.vfhe_cuda_device_faults() == 0, "a bounded device wait gave up during this test"


def has_ifma() -> bool:
    try:
        return "avx512ifma" in Path("/proc/cpuinfo").read_text()
    except OSError:
        return False


os.environ.setdefault("VFHE_CUDA_QUIET", "1")
