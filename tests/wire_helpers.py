"""Host restatement of the compact wire format (vfhe_cuda_pack_rows), for checks."""

from __future__ import annotations

import numpy as np


def pack_rows_host(rows: np.ndarray, bits: list[int]) -> np.ndarray:
    """[B][R][N] uint64 -> [B][bytes] uint8: row r as N fields of bits[r] bits, least
    significant bit first, rows of an item one after another."""
    B, R, N = rows.shape
    assert R == len(bits)
    out = []
    for i in range(B):
        parts = []
        for r, b in enumerate(bits):
            v = rows[i, r].astype(np.uint64)
            if b < 64:
                v = v & np.uint64((1 << b) - 1)
            bitarr = ((v[:, None] >> np.arange(b, dtype=np.uint64)[None, :]) & np.uint64(1)).astype(np.uint8)
            parts.append(np.packbits(bitarr.reshape(-1), bitorder="little"))
        out.append(np.concatenate(parts))
    return np.stack(out)


def unpack_rows_host(packed: np.ndarray, bits: list[int], N: int) -> np.ndarray:
    """[B][bytes] uint8 -> [B][R][N] uint64, the inverse of pack_rows_host."""
    out = []
    for item in packed:
        rows, off = [], 0
        for b in bits:
            nbytes = N * b // 8
            bitarr = np.unpackbits(item[off:off + nbytes], bitorder="little").reshape(N, b).astype(np.uint64)
            rows.append((bitarr << np.arange(b, dtype=np.uint64)[None, :]).sum(axis=1, dtype=np.uint64))
            off += nbytes
        out.append(np.stack(rows))
    return np.stack(out)
