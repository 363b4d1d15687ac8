"""Loading the engine library through cffi (ABI mode).

The cdef is ``include/vfhe_cuda.h`` itself, with its preprocessor lines and the
C++ guard stripped, so the Python binding and the C ABI cannot drift apart.  Part 1
of that header is the reference's cdef surface (modules/*/python/cdef/*.cdef), which
is why the same :class:`Engine` can also wrap another library exporting that surface
(the tests use this for the CPU oracle): the struct prefixes Python dereferences
(``RNS_Polynomial.coeffs``, ``rns_mask``, ``LWE.a`` ...) are identical.

The product engine is the cuda library built by :mod:`vfhe_b200.build`.  Loading it
fails loudly when the library is missing or no CUDA device is usable: there is no
CPU fallback (modules/misc/python/src/_vfhe_native.py:21-56 is the reference's
engine picker this replaces for ``VFHE_ENGINE=cuda``).
"""

from __future__ import annotations

import os
import re
import threading
from pathlib import Path

import cffi

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "vfhe_cuda.h"
CUDA_LIB = Path(__file__).resolve().parent / "lib" / "libvfhe_cuda.so"


class EngineError(RuntimeError):
    """An engine call recorded an error (see ``vfhe_cuda_last_error``)."""


def _cdef_text() -> str:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = []
    skip_cpp = False
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("#ifdef __cplusplus"):
            skip_cpp = True
            continue
        if skip_cpp:
            if s.startswith("#endif"):
                skip_cpp = False
            continue
        if s.startswith("#"):
            continue
        out.append(line)
    # misc.cdef:17 binds libc free() to release safe_aligned_malloc buffers; it is not
    # part of the engine library (the symbol resolves through its libc dependency)
    out.append("void free(void *ptr);")
    return "\n".join(out)


_FFI: cffi.FFI | None = None
_FFI_LOCK = threading.Lock()


def ffi() -> cffi.FFI:
    global _FFI
    with _FFI_LOCK:
        if _FFI is None:
            f = cffi.FFI()
            f.cdef(_cdef_text())
            _FFI = f
        return _FFI


class Engine:
    """One loaded library exporting the vfhe cdef surface."""

    def __init__(self, path: str | os.PathLike, name: str | None = None, check_errors: bool | None = None):
        self.path = str(path)
        self.ffi = ffi()
        self.lib = self.ffi.dlopen(self.path)
        self.name = name or self.ffi.string(self.lib.vfhe_engine_active()).decode()
        # only the cuda engine records errors instead of aborting
        self.check_errors = (self.name == "cuda") if check_errors is None else check_errors

    def check(self, what: str = "") -> None:
        """Raise :class:`EngineError` if the engine recorded an error."""
        if not self.check_errors:
            return
        if self.lib.vfhe_cuda_status() != 0:
            msg = self.ffi.string(self.lib.vfhe_cuda_last_error()).decode()
            self.lib.vfhe_cuda_clear_error()
            raise EngineError(f"{what}: {msg}" if what else msg)

    def __repr__(self) -> str:
        return f"Engine({self.name!r}, {self.path!r})"


_DEFAULT: Engine | None = None
_CUDA: Engine | None = None


def cuda_engine(apply_tuned: bool = True) -> Engine:
    """The B200 engine.  Raises if the library was not built or no GPU is present.
    On first load the tuned transform schedule (vfhe_b200/tuned/, written by
    :mod:`vfhe_b200.autotune`) is applied when present and ``apply_tuned`` is set;
    schedules change launch shapes only, never results."""
    global _CUDA
    if _CUDA is None:
        if not CUDA_LIB.exists():
            raise EngineError(
                f"{CUDA_LIB} is missing: build it with `python -m vfhe_b200.build` "
                "(the cuda engine has no CPU fallback)"
            )
        eng = Engine(CUDA_LIB, "cuda")
        if eng.lib.vfhe_cuda_device() < 0:
            msg = eng.ffi.string(eng.lib.vfhe_cuda_last_error()).decode()
            raise EngineError(f"cuda engine unavailable: {msg}")
        if apply_tuned and not os.environ.get("VFHE_CUDA_NO_TUNED"):
            from . import autotune

            table = autotune.load()
            if table:
                autotune.apply(eng, table)
        _CUDA = eng
    return _CUDA


def default_engine() -> Engine:
    """Engine used by rings created without an explicit ``engine=``."""
    return _DEFAULT if _DEFAULT is not None else cuda_engine()


def set_default_engine(engine: Engine | None) -> None:
    global _DEFAULT
    _DEFAULT = engine


class use_engine:
    """Context manager: ``with use_engine(e): ...`` makes ``e`` the default."""

    def __init__(self, engine: Engine):
        self.engine = engine
        self.prev: Engine | None = None

    def __enter__(self) -> Engine:
        global _DEFAULT
        self.prev = _DEFAULT
        _DEFAULT = self.engine
        return self.engine

    def __exit__(self, *exc) -> None:
        global _DEFAULT
        _DEFAULT = self.prev
