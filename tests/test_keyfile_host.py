"""Evaluation-key file format (vfhe_cuda_keyfile_*), host side, no GPU: round trips of
both element sizes, and every malformed file is refused with a reason."""

from __future__ import annotations

import numpy as np
import pytest

from vfhe_b200 import keyfile
from vfhe_b200.native import EngineError


@pytest.fixture
def eng():
    from vfhe_b200 import build
    from vfhe_b200.native import Engine

    if not build.LIB.exists():
        build.build()
    e = Engine(build.LIB, "cuda")
    yield e
    e.lib.vfhe_cuda_clear_error()


def _ksk(rng, D=3, L=4, N=64):
    primes = [1125899906842597, 1099511627689, 1099511627791, 1125899906842679][:L]
    arr = np.stack([rng.integers(0, q, (D, 2, N), dtype=np.uint64) for q in primes], axis=2)
    return primes, arr


def test_round_trip_u64_and_u32(tmp_path, eng):
    rng = np.random.default_rng(1)
    primes, arr = _ksk(rng)
    p = tmp_path / "rlk.vfhekey"
    h = keyfile.KeyHeader(keyfile.KSK, arr.shape, 8, primes, [0, 1, 64, 0])
    keyfile.write_host(p, h, arr, eng)
    h2, back = keyfile.read_host(p, eng)
    assert np.array_equal(back, arr) and back.dtype == np.uint64
    assert h2.kind == keyfile.KSK and h2.shape == arr.shape and h2.moduli == primes and h2.aux == [0, 1, 64, 0]
    assert p.stat().st_size == 656 + arr.nbytes
    t = rng.integers(0, 1 << 32, (5, 6, 2, 32), dtype=np.uint64).astype(np.uint32)
    q = tmp_path / "bsk.vfhekey"
    keyfile.write_host(q, keyfile.KeyHeader(keyfile.TORUS_BSK, t.shape, 4, [], [7, 3, 0, 0]), t, eng)
    h3, t2 = keyfile.read_host(q, eng)
    assert np.array_equal(t2, t) and t2.dtype == np.uint32 and h3.aux[:2] == [7, 3]


def _raw(path):
    return bytearray(path.read_bytes())


def test_corruptions_are_refused(tmp_path, eng):
    rng = np.random.default_rng(2)
    primes, arr = _ksk(rng, D=2, L=2, N=32)
    good = tmp_path / "k.vfhekey"
    keyfile.write_host(good, keyfile.KeyHeader(keyfile.KSK, arr.shape, 8, primes), arr, eng)
    base = _raw(good)
    cases = {
        "magic": lambda b: b.__setitem__(0, ord("X")),
        "version": lambda b: b.__setitem__(8, 2),
        "payload bit": lambda b: b.__setitem__(700, b[700] ^ 1),
        "shape": lambda b: b.__setitem__(24, b[24] + 1),
    }
    for name, mutate in cases.items():
        b = bytearray(base)
        mutate(b)
        bad = tmp_path / f"bad_{name.replace(' ', '_')}.vfhekey"
        bad.write_bytes(bytes(b))
        with pytest.raises(EngineError):
            keyfile.read_host(bad, eng)
    trunc = tmp_path / "trunc.vfhekey"
    trunc.write_bytes(bytes(base[:-8]))
    with pytest.raises(EngineError, match="truncated|payload"):
        keyfile.read_host(trunc, eng)
    extra = tmp_path / "extra.vfhekey"
    extra.write_bytes(bytes(base) + b"\0")
    with pytest.raises(EngineError):
        keyfile.read_host(extra, eng)
    short = tmp_path / "short.vfhekey"
    short.write_bytes(bytes(base[:100]))
    with pytest.raises(EngineError):
        keyfile.read_header(short, eng)


def test_refuses_bad_headers_and_small_buffers(tmp_path, eng):
    rng = np.random.default_rng(3)
    primes, arr = _ksk(rng, D=1, L=2, N=16)
    with pytest.raises(ValueError):
        keyfile.write_host(tmp_path / "x", keyfile.KeyHeader(keyfile.KSK, (9,), 8, primes), arr, eng)
    p = tmp_path / "k.vfhekey"
    keyfile.write_host(p, keyfile.KeyHeader(keyfile.KSK, arr.shape, 8, primes), arr, eng)
    h = eng.ffi.new("VfheKeyHeader*")
    small = np.empty(arr.size - 1, dtype=np.uint64)
    assert eng.lib.vfhe_cuda_keyfile_read(bytes(str(p), "utf8"), h, eng.ffi.from_buffer(small), small.nbytes) == 1
    assert b"smaller" in eng.ffi.string(eng.lib.vfhe_cuda_last_error())
    eng.lib.vfhe_cuda_clear_error()
    bad = eng.ffi.new("VfheKeyHeader*")
    bad.kind, bad.elem_bytes, bad.ndims = 1, 3, 1
    bad.dims[0] = 4
    assert eng.lib.vfhe_cuda_keyfile_payload_bytes(bad) == 0
