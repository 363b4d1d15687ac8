"""numpy <-> ctypes glue for the exact torus CGGI oracle (tests only)."""

from __future__ import annotations

import ctypes

import numpy as np


def u32p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def oracle_bootstrap(lib, lwe: np.ndarray, tv: np.ndarray, bsk: np.ndarray, params) -> np.ndarray:
    """Exact blind rotation + extraction of each row of lwe [B][n+1] -> [B][N+1]."""
    p = params
    bsk = np.ascontiguousarray(bsk, dtype=np.uint32)
    tv = np.ascontiguousarray(tv, dtype=np.uint32)
    out = np.zeros((lwe.shape[0], p.N + 1), dtype=np.uint32)
    for b in range(lwe.shape[0]):
        row = np.ascontiguousarray(lwe[b, :p.n], dtype=np.uint32)
        o = np.zeros(p.N + 1, dtype=np.uint32)
        lib.tor_bootstrap(u32p(o), u32p(row), int(lwe[b, p.n]), u32p(tv), u32p(bsk), p.n, p.N, p.bs_base_log,
                          p.bs_levels, p.t)
        out[b] = o
    return out


def oracle_keyswitch(lib, ext: np.ndarray, ksk: np.ndarray, params) -> np.ndarray:
    p = params
    ksk = np.ascontiguousarray(ksk, dtype=np.uint32)
    out = np.zeros((ext.shape[0], p.n + 1), dtype=np.uint32)
    for b in range(ext.shape[0]):
        o = np.zeros(p.n + 1, dtype=np.uint32)
        lib.tor_keyswitch(u32p(o), u32p(np.ascontiguousarray(ext[b], dtype=np.uint32)), u32p(ksk), p.N, p.n,
                          p.ks_base_log, p.ks_levels)
        out[b] = o
    return out


def oracle_external_product(lib, c: np.ndarray, ggsw: np.ndarray, params) -> np.ndarray:
    p = params
    out = np.zeros(2 * p.N, dtype=np.uint32)
    lib.tor_external_product(u32p(out), u32p(np.ascontiguousarray(c, dtype=np.uint32)),
                             u32p(np.ascontiguousarray(ggsw, dtype=np.uint32)), p.N, p.bs_base_log, p.bs_levels)
    return out


def torus_distance(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    d = (x.astype(np.int64) - y.astype(np.int64)) & 0xFFFFFFFF
    return np.minimum(d, (1 << 32) - d)
