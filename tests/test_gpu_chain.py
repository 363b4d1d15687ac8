"""NTT -> product -> INTT chains in one kernel (chain.cu, behind
vfhe_cuda_ntt_mul_intt_batch).

Every (P, split) the fused kernel takes must give the residues of the same chain run as
separate launches (vfhe_cuda_ntt_batch forward twice, vfhe_cuda_poly_mul_batch,
vfhe_cuda_ntt_batch inverse), bit for bit, including the wrap terms of the incomplete
product at split > 1 and canonical extremes; one shape is also checked against the
oracle engine through the reference API (polynomial_RNSc_to_RNS, polynomial_mul_RNS_polynomial,
polynomial_RNS_to_RNSc).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(ring, B, rng, extremes=False):
    x = np.stack([np.stack([rng.integers(0, q, ring.N, dtype=np.uint64) for q in ring.primes]) for _ in range(B)])
    if extremes:
        x[0, :, :8] = 0
        x[0, :, 8:16] = np.array(ring.primes, dtype=np.uint64)[:, None] - 1
    return x


def _separate_launches(cuda, ring, ta, tb):
    import torch

    ffi, lib = cuda.ffi, cuda.lib
    st = ffi.cast("void*", torch.cuda.current_stream().cuda_stream)
    B, L = ta.shape[0], ta.shape[1]
    limbs = ffi.new("uint32_t[]", ring.prime_indices[:L])
    a, b = ta.clone(), tb.clone()
    p = lambda t: ffi.cast("uint64_t*", t.data_ptr())  # noqa: E731
    assert lib.vfhe_cuda_ntt_batch(ring.NTT, 0, p(a), p(a), B, limbs, L, st) == 0
    assert lib.vfhe_cuda_ntt_batch(ring.NTT, 0, p(b), p(b), B, limbs, L, st) == 0
    assert lib.vfhe_cuda_poly_mul_batch(ring.NTT, p(a), p(a), p(b), B, limbs, L, st) == 0
    assert lib.vfhe_cuda_ntt_batch(ring.NTT, 1, p(a), p(a), B, limbs, L, st) == 0
    torch.cuda.synchronize()
    return a.cpu().numpy().view(np.uint64)


def _chain(cuda, ring, ta, tb):
    import torch

    ffi, lib = cuda.ffi, cuda.lib
    st = ffi.cast("void*", torch.cuda.current_stream().cuda_stream)
    B, L = ta.shape[0], ta.shape[1]
    limbs = ffi.new("uint32_t[]", ring.prime_indices[:L])
    out = torch.empty_like(ta)
    p = lambda t: ffi.cast("uint64_t*", t.data_ptr())  # noqa: E731
    n0 = lib.vfhe_cuda_launch_count()
    rc = lib.vfhe_cuda_ntt_mul_intt_batch(ring.NTT, p(out), p(ta), p(tb), B, limbs, L, st)
    assert rc == 0, ffi.string(lib.vfhe_cuda_last_error()).decode()
    launches = lib.vfhe_cuda_launch_count() - n0
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint64), launches


@pytest.mark.parametrize("N,split,sizes,B", [
    (512, 1, [50, 45], 3), (1024, 1, [50], 5), (1024, 2, [50, 40], 2), (2048, 2, [50, 49, 30], 3),
    (2048, 4, [50, 50], 4), (4096, 1, [50, 50, 50], 64), (4096, 2, [50, 36], 3), (4096, 4, [50, 50, 50], 64),
    (4096, 8, [50, 48], 2), (8192, 1, [50, 40, 40], 2), (8192, 2, [49, 50], 2), (8192, 4, [50, 44], 3),
    (8192, 8, [50, 50], 2),
])
def test_chain_kernel_matches_separate_launches(cuda, N, split, sizes, B):
    from vfhe_b200.arith import Ring
    from vfhe_b200.batch import to_device

    ring = Ring(N, prime_size=sizes, split_degree=split, engine=cuda)
    assert ring.split_degree == split
    rng = np.random.default_rng(N * 10 + split)
    ta = to_device(_rows(ring, B, rng, extremes=True))
    tb = to_device(_rows(ring, B, rng, extremes=True))
    want = _separate_launches(cuda, ring, ta, tb)
    got, launches = _chain(cuda, ring, ta, tb)
    assert launches == 1, "the chain should be one kernel at this shape"
    assert np.array_equal(got, want), (N, split)
    cuda.check("chain")


def test_chain_config0_matches_oracle(cuda, oracle_engine):
    """64 pairs at N = 4096, L = 3 (50-bit primes), split 4: the fused chain against the
    oracle engine running the reference API chain on the same rows."""
    from tests.helpers import poly_from_rows, twin_rings
    from vfhe_b200.arith import repr
    from vfhe_b200.batch import to_device

    rg, ro = twin_rings([cuda, oracle_engine], 4096, [50, 50, 50], split=4)
    rng = np.random.default_rng(2026)
    A, Bv = _rows(rg, 64, rng), _rows(rg, 64, rng)
    got, launches = _chain(cuda, rg, to_device(A), to_device(Bv))
    assert launches == 1
    for i in range(0, 64, 9):  # a spread of the pairs on the CPU oracle
        pa, pb = poly_from_rows(ro, A[i]), poly_from_rows(ro, Bv[i])
        pa.to_NTT()
        pb.to_NTT()
        prod = pa * pb
        prod.to_repr(repr.coeff)
        assert np.array_equal(prod.rows(), got[i]), i


def test_chain_falls_back_for_other_shapes(cuda):
    """Shapes outside the fused kernel (N = 2^14, or rows not 16-byte aligned) take the
    separate launches and still agree with them."""
    import torch

    from vfhe_b200.arith import Ring
    from vfhe_b200.batch import to_device

    ring = Ring(2**14, prime_size=[50, 40], split_degree=1, engine=cuda)
    rng = np.random.default_rng(5)
    ta, tb = to_device(_rows(ring, 2, rng)), to_device(_rows(ring, 2, rng))
    got, launches = _chain(cuda, ring, ta, tb)
    assert launches > 1
    assert np.array_equal(got, _separate_launches(cuda, ring, ta, tb))

    small = Ring(4096, prime_size=[50], split_degree=4, engine=cuda)
    flat_a = to_device(np.concatenate([[0], _rows(small, 1, rng).ravel()]).astype(np.uint64))
    flat_b = to_device(np.concatenate([[0], _rows(small, 1, rng).ravel()]).astype(np.uint64))
    ua, ub = flat_a[1:].view(1, 1, 4096), flat_b[1:].view(1, 1, 4096)  # 8-byte, not 16-byte aligned
    ffi, lib = cuda.ffi, cuda.lib
    out = torch.empty(1 + 4096, dtype=torch.int64, device="cuda")[1:].view(1, 1, 4096)
    limbs = ffi.new("uint32_t[]", small.prime_indices)
    p = lambda t: ffi.cast("uint64_t*", t.data_ptr())  # noqa: E731
    st = ffi.cast("void*", torch.cuda.current_stream().cuda_stream)
    n0 = lib.vfhe_cuda_launch_count()
    assert lib.vfhe_cuda_ntt_mul_intt_batch(small.NTT, p(out), p(ua), p(ub), 1, limbs, 1, st) == 0
    assert lib.vfhe_cuda_launch_count() - n0 > 1
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint64),
                          _separate_launches(cuda, small, ua.contiguous(), ub.contiguous()))
