"""The compact wire format's host side, without a GPU: the size the library reports
for a layout, its refusal of layouts that are not whole 64-bit words, and the numpy
restatement that the GPU tests check the kernels against (a round trip here)."""

from __future__ import annotations

import numpy as np
import pytest

from tests.wire_helpers import pack_rows_host, unpack_rows_host


@pytest.fixture(scope="module")
def lib_engine():
    from vfhe_b200 import build
    from vfhe_b200.native import Engine

    if not build.LIB.exists():
        build.build()
    return Engine(build.LIB)


def test_packed_bytes(lib_engine):
    ffi, lib = lib_engine.ffi, lib_engine.lib
    bits = ffi.new("uint32_t[]", ([50] + [40] * 8) * 2)
    assert lib.vfhe_cuda_packed_bytes(1 << 14, bits, 18, 256) == 256 * (1 << 14) * 740 // 8
    lib_engine.check("valid layout")
    odd = ffi.new("uint32_t[]", [33])
    assert lib.vfhe_cuda_packed_bytes(32, odd, 1, 1) == 0
    assert lib.vfhe_cuda_status() != 0
    lib.vfhe_cuda_clear_error()
    assert lib.vfhe_cuda_packed_bytes(64, ffi.new("uint32_t[]", [0]), 1, 1) == 0
    lib.vfhe_cuda_clear_error()
    assert lib.vfhe_cuda_packed_bytes(64, bits, 129, 1) == 0
    lib.vfhe_cuda_clear_error()


@pytest.mark.parametrize("bits,N", [([50, 40, 40], 64), ([1, 7, 13, 31, 33, 63, 64, 8], 64), ([37, 41], 128)])
def test_host_packer_round_trip(bits, N):
    rng = np.random.default_rng(N + len(bits))
    rows = np.stack([np.stack([rng.integers(0, 1 << b, N, dtype=np.uint64) if b < 64
                               else rng.integers(0, 2**64, N, dtype=np.uint64) for b in bits]) for _ in range(3)])
    packed = pack_rows_host(rows, bits)
    assert packed.shape == (3, N * sum(bits) // 8)
    assert np.array_equal(unpack_rows_host(packed, bits, N), rows)


def test_host_packer_bit_order():
    """Residue x of a row occupies bits [x b, x b + b), least significant bit first."""
    rows = np.array([[[1, 2, 3, 4, 5, 6, 7, 8]]], dtype=np.uint64)
    assert pack_rows_host(rows, [8]).tolist() == [[1, 2, 3, 4, 5, 6, 7, 8]]
    rows = np.array([[[0b101] + [0] * 63]], dtype=np.uint64)
    assert pack_rows_host(rows, [3])[0, 0] == 0b101


@pytest.mark.parametrize("bits,N,items,threads", [
    ([50, 40, 40], 64, 3, 1),
    ([1, 7, 13, 31, 33, 63, 64, 8], 64, 2, 3),
    ([37, 41], 128, 5, 0),
    ([50] + [40] * 8, 1024, 4, 4),  # one ciphertext component of the CKKS benchmark's chain
])
def test_native_host_packer_matches_format(lib_engine, bits, N, items, threads):
    """vfhe_cuda_pack_rows_host / _unpack_rows_host (the sender's and receiver's side on
    the host) write and read exactly the format the numpy restatement defines, for any
    thread count, with residues wider than their field masked as the GPU packer does."""
    from vfhe_b200.batch import WireFormat

    rng = np.random.default_rng(N * items + len(bits))
    rows = np.stack([np.stack([rng.integers(0, 2**63, N, dtype=np.uint64) for _ in bits]) for _ in range(items)])
    masked = rows.copy()
    for r, b in enumerate(bits):
        if b < 64:
            masked[:, r] &= np.uint64((1 << b) - 1)
    wf = WireFormat(N, bits, engine=lib_engine)
    packed = wf.pack_host(rows, nthreads=threads)
    assert np.array_equal(packed, pack_rows_host(masked, bits))
    back = np.empty_like(rows)
    wf.unpack_host(packed, back, nthreads=threads)
    assert np.array_equal(back, masked)
    lib_engine.check("host packer")


def test_native_host_packer_refuses_bad_layouts(lib_engine):
    """The host packer checks its layout and buffers like the GPU one and records an
    error instead of writing anything."""
    ffi, lib = lib_engine.ffi, lib_engine.lib
    rows = np.zeros((1, 1, 64), dtype=np.uint64)
    out = np.full(64, 7, dtype=np.uint8)
    pr = ffi.cast("uint64_t*", rows.ctypes.data)
    po = ffi.cast("void*", out.ctypes.data)
    for bits, items, dst, src in (([33], 1, po, pr), ([0], 1, po, pr), ([40], 1, ffi.NULL, pr),
                                  ([40], 1, po, ffi.NULL), ([40], 0, po, pr)):
        lib.vfhe_cuda_clear_error()
        b = ffi.new("uint32_t[]", bits)
        N = 32 if bits == [33] else 64
        assert lib.vfhe_cuda_pack_rows_host(dst, src, N, b, 1, items, 1) != 0
        assert lib.vfhe_cuda_status() != 0
        lib.vfhe_cuda_clear_error()
        assert lib.vfhe_cuda_unpack_rows_host(ffi.cast("uint64_t*", src) if src != ffi.NULL else ffi.NULL,
                                              dst, N, b, 1, items, 1) != 0
        lib.vfhe_cuda_clear_error()
    assert (out == 7).all()


def test_native_host_packer_every_fixed_width(lib_engine):
    """Every field width the host packer has a fixed-width form for (24..62), and its
    neighbours on either side that take the general loop, against the numpy restatement:
    several periods of each width, several items, one and four threads."""
    from vfhe_b200.batch import WireFormat

    rng = np.random.default_rng(23)
    N = 256  # a multiple of every width's period (64 / gcd(64, b) divides 64)
    for b in range(22, 65):
        bits = [b, b]
        rows = np.stack([np.stack([rng.integers(0, 2**64 - 1, N, dtype=np.uint64, endpoint=True) for _ in bits])
                         for _ in range(3)])
        masked = rows & np.uint64((1 << b) - 1) if b < 64 else rows.copy()
        wf = WireFormat(N, bits, engine=lib_engine)
        for threads in (1, 4):
            packed = wf.pack_host(rows, nthreads=threads)
            assert np.array_equal(packed, pack_rows_host(masked, bits)), (b, threads)
            back = np.empty_like(rows)
            wf.unpack_host(packed, back, nthreads=threads)
            assert np.array_equal(back, masked), (b, threads)
    lib_engine.check("host packer")
