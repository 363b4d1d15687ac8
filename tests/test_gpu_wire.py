"""The compact wire format of residue rows (vfhe_cuda_pack_rows / unpack_rows): bit for
bit against a numpy packer written from the format's definition, round trips at the
CKKS benchmark's ring, and the size checks of the host side."""

from __future__ import annotations

import numpy as np
import pytest

from tests.wire_helpers import pack_rows_host

pytestmark = pytest.mark.gpu


def _rows(rng, B, bits, N):
    return np.stack([np.stack([rng.integers(0, 1 << b, N, dtype=np.uint64) if b < 64
                               else rng.integers(0, 2**64, N, dtype=np.uint64) for b in bits]) for _ in range(B)])


@pytest.mark.parametrize("bits,N,B", [
    ([50, 40, 40, 40], 64, 3),
    ([1, 7, 13, 31, 33, 63, 64, 8], 64, 2),
    ([37, 41], 128, 5),
    ([50] + [40] * 8, 256, 2),
])
def test_pack_matches_host_packer(cuda, bits, N, B):
    import torch

    from vfhe_b200.batch import WireFormat, to_device

    rng = np.random.default_rng(sum(bits) + N)
    rows = _rows(rng, B, bits, N)
    wf = WireFormat(N, bits, cuda)
    assert wf.item_bytes == N * sum(bits) // 8
    d = to_device(rows)
    packed = wf.pack(d)
    torch.cuda.synchronize()
    ref = pack_rows_host(rows, bits)
    assert np.array_equal(packed.cpu().numpy(), ref)
    back = wf.unpack(torch.from_numpy(ref).cuda(), (B, len(bits), N))
    torch.cuda.synchronize()
    assert np.array_equal(back.cpu().numpy().view(np.uint64), rows)


def test_round_trip_ckks_ring(cuda):
    """A [B][2][9][2^14] ciphertext batch at one 50-bit and eight 40-bit primes."""
    import torch

    from vfhe_b200.batch import WireFormat

    N, B = 1 << 14, 6
    bits = ([50] + [40] * 8) * 2
    wf = WireFormat(N, bits, cuda)
    assert wf.item_bytes == N * 370 * 2 // 8
    g = torch.Generator(device="cuda").manual_seed(5)
    lim = torch.tensor([(1 << b) for b in bits], dtype=torch.float64, device="cuda").view(1, 2, 9, 1)
    u = torch.rand((B, 2, 9, N), generator=g, device="cuda", dtype=torch.float64)
    ct = (u * lim).to(torch.int64)
    packed = wf.pack(ct)
    assert packed.shape == (B, wf.item_bytes)
    back = wf.unpack(packed, ct.shape)
    torch.cuda.synchronize()
    assert torch.equal(back, ct)


def test_size_checks(cuda):
    """Bad shapes are refused with a recorded error (read and cleared here, so no later
    call sees it)."""
    from vfhe_b200.native import EngineError

    ffi, lib = cuda.ffi, cuda.lib
    bits = ffi.new("uint32_t[]", [40, 33])
    assert lib.vfhe_cuda_packed_bytes(64, bits, 2, 3) == 3 * 64 * 73 // 8
    cuda.check("valid shape")
    assert lib.vfhe_cuda_packed_bytes(32, bits, 2, 1) == 0  # 32 * 33 bits is not whole words
    with pytest.raises(EngineError, match="multiple of 64"):
        cuda.check()
    bad = ffi.new("uint32_t[]", [65])
    assert lib.vfhe_cuda_packed_bytes(64, bad, 1, 1) == 0
    with pytest.raises(EngineError, match="1..64"):
        cuda.check()
    assert lib.vfhe_cuda_pack_rows(ffi.NULL, ffi.NULL, 64, bits, 2, 1, ffi.NULL) != 0
    with pytest.raises(EngineError, match="null buffers"):
        cuda.check()
    assert lib.vfhe_cuda_status() == 0
