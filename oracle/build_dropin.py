"""Build the reference's own Python front end over several engines -- TEST INFRASTRUCTURE.

The drop-in claim of the cuda engine is that the reference's unchanged Python
(`vfhe.arith`, `vfhe.mlwe`, `vfhe.fhe`) runs on it once the engine is registered.  This
recipe builds exactly what the reference's own build would install for that
(meson.build:130-246, tools/meson/generate_ffi_c.py:37-47), without running meson:

  oracle/_ref/dropin/modules/...   the reference's Python sources and test suites,
                                   copied verbatim from the checkout (git-ignored output;
                                   copied so the tree travels with the build outputs)
  oracle/_ref/dropin/smoke/ckks.py the reference's CKKS smoke script, verbatim
  oracle/_ref/dropin/build/
      _vfhe_cpu                    the CPU probe extension (vfhe_cpu.cdef + cpu_probe.c)
      _vfhe_native_cuda            API mode: the five reference cdefs compiled against
                                   include/vfhe_cuda.h, linked to vfhe_b200/lib/libvfhe_cuda.so
      _vfhe_native_<engine>        the same cdefs against the reference's own headers,
                                   linked to oracle/_ref/libvfhe_ref_<engine>.so (portable,
                                   and avx512ifma when the compiler has the ISA)
      _vfhe_engines.py             the picker's table, cuda first (requires None)

Only tests load these outputs.  Run `python oracle/build_dropin.py` after
`oracle/build_ref.sh` and `python -m vfhe_b200.build`; it does nothing when the reference
checkout is absent (the prebuilt tree is used as it is).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
REF = Path(os.environ.get("VFHE_REFERENCE_ROOT", "/root/reference"))
OUT = HERE / "_ref" / "dropin"
BUILD = OUT / "build"

CDEFS = [
    "modules/arith/python/cdef/arith.cdef",
    "modules/misc/python/cdef/misc.cdef",
    "modules/misc/python/cdef/vfhe_cpu.cdef",
    "modules/mlwe/python/cdef/mlwe.cdef",
    "modules/fhe/python/cdef/fhe.cdef",
]
PY_MODULES = ["arith", "misc", "mlwe", "fhe"]


def _copy_python() -> None:
    for m in PY_MODULES:
        for part in ("src", "test"):
            src = REF / "modules" / m / "python" / part
            dst = OUT / "modules" / m / "python" / part
            if dst.exists():
                shutil.rmtree(dst)
            if src.is_dir():
                shutil.copytree(src, dst, ignore=shutil.ignore_patterns("__pycache__"))
    shutil.copy2(REF / "modules" / "conftest.py", OUT / "modules" / "conftest.py")
    (OUT / "smoke").mkdir(parents=True, exist_ok=True)
    shutil.copy2(REF / "smoke" / "ckks.py", OUT / "smoke" / "ckks.py")


def _ffi_build(name: str, source: str, **kw) -> None:
    import cffi

    ffi = cffi.FFI()
    ffi.cdef("\n".join((REF / c).read_text() for c in CDEFS) if name != "_vfhe_cpu"
             else (REF / "modules/misc/python/cdef/vfhe_cpu.cdef").read_text())
    ffi.set_source(name, source, **kw)
    tmp = BUILD / ("_tmp_" + name)
    tmp.mkdir(parents=True, exist_ok=True)
    so = ffi.compile(tmpdir=str(tmp), verbose=False)
    shutil.move(so, BUILD / Path(so).name)
    shutil.rmtree(tmp)


def _have_ifma() -> bool:
    r = subprocess.run(["gcc", "-mavx512f", "-mavx512ifma", "-x", "c", "-", "-o", os.devnull],
                       input="int main(void){return 0;}", capture_output=True, text=True)
    return r.returncode == 0


def build() -> Path:
    if not (REF / "modules").is_dir():
        print(f"build_dropin: no reference checkout at {REF}; keeping {OUT}", file=sys.stderr)
        return OUT
    cuda_lib = REPO / "vfhe_b200" / "lib" / "libvfhe_cuda.so"
    if not cuda_lib.exists():
        raise SystemExit("build_dropin: build the cuda engine first (python -m vfhe_b200.build)")
    if BUILD.exists():
        shutil.rmtree(BUILD)
    BUILD.mkdir(parents=True)
    _copy_python()

    m = REF / "modules"
    ref_inc = [str(m / "arith/c/include"), str(m / "arith/c/src"), str(m / "misc/c/include"),
               str(m / "mlwe/c/include"), str(HERE / "blake3_standin")]
    # the CPU probe: the reference's own translation unit
    _ffi_build("_vfhe_cpu", '#include "vfhe_cpu.h"', sources=[str(m / "misc/c/src/cpu_probe.c")],
               include_dirs=ref_inc)
    # the cuda engine: reference cdefs, this repository's header, the engine library
    _ffi_build("_vfhe_native_cuda", '#include "vfhe_cuda.h"\n#include <stdlib.h>',
               include_dirs=[str(REPO / "include")], libraries=["vfhe_cuda"],
               library_dirs=[str(cuda_lib.parent)],
               extra_link_args=["-Wl,-rpath,$ORIGIN/../../../../vfhe_b200/lib"])
    engines = [("cuda", None)]
    # the headers meson.build hands the reference's own ffi generator (the modules'
    # meson.build header_files)
    headers = "\n".join(f'#include "{h}"' for h in ("arith.h", "misc.h", "mlwe.h", "rns-rlwe.h"))
    for name, cflags in (("avx512ifma", ["-mavx512f", "-mavx512ifma", "-mavx512dq", "-mavx512vl", "-mavx2"]),
                         ("portable", ["-DPORTABLE_BUILD"])):
        lib = HERE / "_ref" / f"libvfhe_ref_{name}.so"
        if not lib.exists() or (name == "avx512ifma" and not _have_ifma()):
            continue
        _ffi_build(f"_vfhe_native_{name}", headers + "\n#include <stdlib.h>", include_dirs=ref_inc,
                   libraries=[f"vfhe_ref_{name}"], library_dirs=[str(lib.parent)],
                   extra_compile_args=cflags + ["-w"], extra_link_args=["-Wl,-rpath,$ORIGIN/../.."])
        engines.append((name, "avx512ifma" if name == "avx512ifma" else None))
    rows = ",\n".join(f"    ({n!r}, {r!r})" for n, r in engines)
    (BUILD / "_vfhe_engines.py").write_text(
        "# Engine table for the drop-in tests (the reference's picker reads it).\n"
        f"ENGINES = [\n{rows},\n]\n")
    print(f"built {OUT} with engines {[n for n, _ in engines]}")
    return OUT


def pythonpath() -> str:
    """PYTHONPATH under which the reference's own `import vfhe` resolves to the copied
    sources and `_vfhe_native` to the extensions built here."""
    parts = [str(BUILD)] + [str(OUT / "modules" / m / "python" / "src") for m in PY_MODULES]
    return os.pathsep.join(parts)


if __name__ == "__main__":
    build()
