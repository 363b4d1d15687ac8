"""Empty batches through the batched device API: every batched compute call given an
empty batch returns success without launching anything, once its pool and limb list
check out, and still reports a bad limb list as an error.  The Python wrappers pass
empty tensors straight through."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ring(cuda):
    from vfhe_b200.arith import Ring

    return Ring(2**12, prime_size=[50, 40, 40, 50], split_degree=1, engine=cuda)


def _calls(cuda, ring, buf, limbs, nl, bad=False):
    """(name, thunk) for every batched compute entry point with batch 0."""
    ffi, lib = cuda.ffi, cuda.lib
    p = ffi.cast("uint64_t*", buf.data_ptr())
    st = ffi.NULL
    special = ring.prime_indices[-1] if not bad else 1000
    ws = ffi.cast("void*", buf.data_ptr())
    gens = ffi.new("uint64_t[]", [5])
    keys = ffi.new("uint64_t*[]", [p])
    factors = ffi.new("uint64_t[]", [1] * 8)
    return [
        ("poly_mul", lambda: lib.vfhe_cuda_poly_mul_batch(ring.NTT, p, p, p, 0, limbs, nl, st)),
        ("ntt_mul_intt", lambda: lib.vfhe_cuda_ntt_mul_intt_batch(ring.NTT, p, p, p, 0, limbs, nl, st)),
        ("ckks_mul", lambda: lib.vfhe_cuda_ckks_mul_relin_rescale_batch(ring.NTT, p, p, p, 0, limbs, nl, special, p,
                                                                        ws, st)),
        ("ckks_rotate", lambda: lib.vfhe_cuda_ckks_rotate_batch(ring.NTT, p, p, 0, limbs, nl, special, gens, keys, ws,
                                                                st)),
        ("keyswitch", lambda: lib.vfhe_cuda_keyswitch_batch(ring.NTT, p, p, 0, limbs, nl, special, p, ws, st)),
        ("encrypt", lambda: lib.vfhe_cuda_rlwe_encrypt_batch(ring.NTT, p, p, 0, limbs, nl, p, 3.2, st)),
        ("gen_ksk", lambda: lib.vfhe_cuda_gen_ksk_batch(ring.NTT, p, p, 0, limbs, nl, factors, p, 3.2, st)),
        ("cggi", lambda: lib.vfhe_cuda_cggi_bootstrap_batch(ring.NTT, p, p, p, p, 0, 630, limbs, min(nl, 2), special,
                                                            p, p, 16, ws, st)),
    ]


def test_empty_batches_are_no_ops(cuda, ring):
    import torch

    ffi, lib = cuda.ffi, cuda.lib
    buf = torch.zeros(1 << 16, dtype=torch.int64, device="cuda")
    before = buf.clone()
    limbs = ffi.new("uint32_t[]", ring.prime_indices[:3])
    lib.vfhe_cuda_clear_error()
    n0 = lib.vfhe_cuda_launch_count()
    for name, call in _calls(cuda, ring, buf, limbs, 3):
        assert call() == 0, (name, ffi.string(lib.vfhe_cuda_last_error()).decode())
        assert lib.vfhe_cuda_status() == 0, name
    torch.cuda.synchronize()
    assert lib.vfhe_cuda_launch_count() == n0  # nothing was launched
    assert torch.equal(buf, before)  # and nothing was written


def test_empty_batch_still_checks_limbs(cuda, ring):
    import torch

    ffi, lib = cuda.ffi, cuda.lib
    buf = torch.zeros(1 << 16, dtype=torch.int64, device="cuda")
    bad = ffi.new("uint32_t[]", [ring.prime_indices[0], 1000, ring.prime_indices[1]])
    for name, call in _calls(cuda, ring, buf, bad, 3):
        lib.vfhe_cuda_clear_error()
        assert call() != 0, name
        assert "limb" in ffi.string(lib.vfhe_cuda_last_error()).decode(), name
    lib.vfhe_cuda_clear_error()


def test_empty_ckks_batches_through_the_wrappers(cuda):
    import torch

    from vfhe_b200.batch import CkksBatch, key_tensor
    from tests.test_gpu_batch import _setup

    s, key, rlk, gks, cts = _setup(cuda, 2**12, 3, 2, [1], seed=3)
    special = s.special_rings[0].prime_indices[-1]
    L, N = len(s.rings[0].primes), 2**12
    empty = torch.empty((0, 2, L, N), dtype=torch.int64, device="cuda")
    out = CkksBatch(s.rings[0], special).mul_relin_rescale(empty, empty, key_tensor(rlk))
    assert tuple(out.shape) == (0, 2, L - 1, N)
    rot = CkksBatch(s.rings[1], special).rotate(out, [], [])
    torch.cuda.synchronize()
    assert tuple(rot.shape) == (0, 2, L - 1, N)
    assert cuda.lib.vfhe_cuda_status() == 0
    _ = np
