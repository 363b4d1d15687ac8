"""The C-ABI library loads without a GPU and exports every function include/*.h declares."""

from __future__ import annotations

import ctypes
from pathlib import Path

import pycparser
from pycparser import c_ast

ROOT = Path(__file__).resolve().parent.parent
FAKE_TYPEDEFS = "typedef unsigned long uint64_t; typedef long int64_t; typedef unsigned int uint32_t; " \
                "typedef int int32_t; typedef unsigned char uint8_t; typedef unsigned long size_t; typedef _Bool bool;\n"


def declared_functions(header: Path) -> list[str]:
    from vfhe_b200 import native

    text = native._cdef_text() if header == native.HEADER else header.read_text()
    ast = pycparser.CParser().parse(FAKE_TYPEDEFS + text, filename=str(header))
    names = []
    for node in ast.ext:
        if isinstance(node, c_ast.Decl) and isinstance(node.type, c_ast.FuncDecl):
            names.append(node.name)
    return names


def built_library() -> Path:
    from vfhe_b200 import build

    if not build.LIB.exists():
        build.build()
    return build.LIB


def test_header_parses_and_is_nontrivial():
    names = declared_functions(ROOT / "include" / "vfhe_cuda.h")
    assert len(names) > 150
    for must in ("polynomial_RNSc_to_RNS", "mlwe_RNSc_GHS_hybrid_keyswitch", "mgsw_CMUX", "vfhe_cuda_ntt_batch",
                 "vfhe_cuda_ckks_mul_relin_rescale_batch", "vfhe_cuda_worklist_run", "vfhe_cuda_cggi_bootstrap_batch"):
        assert must in names


def test_library_exports_every_declared_function():
    lib = ctypes.CDLL(str(built_library()))
    missing = [n for n in declared_functions(ROOT / "include" / "vfhe_cuda.h") if not hasattr(lib, n)]
    assert missing == []


def test_engine_name_without_gpu():
    lib = ctypes.CDLL(str(built_library()))
    lib.vfhe_engine_active.restype = ctypes.c_char_p
    assert lib.vfhe_engine_active() == b"cuda"
