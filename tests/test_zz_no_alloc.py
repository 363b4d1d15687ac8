"""The allocation-free NTT -> product -> INTT entry point.

vfhe_cuda_ntt_mul_intt_batch_noalloc serves callers that cannot let the library
allocate GPU memory (stream-capture code, host runtimes that own device memory,
allocation-free serving loops); its scratch is a static device array.  Its output
must equal vfhe_cuda_ntt_mul_intt_batch's, bit for bit, call after call (the second
call also shows the shared scratch keeps no stale state that matters).  This file is
named to be collected last.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(cuda, fn_name, ring, a, b):
    import torch

    ffi = cuda.ffi
    out = torch.empty_like(a)
    limbs = ffi.new("uint32_t[]", ring.prime_indices)
    p = lambda t: ffi.cast("uint64_t*", t.data_ptr())  # noqa: E731
    st = ffi.cast("void*", torch.cuda.current_stream().cuda_stream)
    rc = getattr(cuda.lib, fn_name)(ring.NTT, p(out), p(a), p(b), a.shape[0], limbs, ring.ell, st)
    torch.cuda.synchronize()
    assert rc == 0, ffi.string(cuda.lib.vfhe_cuda_last_error()).decode()
    return out.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("N,sizes,split,batch", [
    (4096, [50, 50, 50], None, 64),   # 64 pairs at the NTT round-trip configuration: 786,432 residues
    (2**14, [50] + [40] * 8 + [50], 1, 2),
    (2**16, [50] * 4, 1, 3),
])
def test_noalloc_matches_allocating_entry(cuda, N, sizes, split, batch):
    from vfhe_b200.arith import Ring
    from vfhe_b200.batch import to_device

    ring = Ring(N, prime_size=sizes, split_degree=split, engine=cuda)
    rng = np.random.default_rng(N + batch)
    for _ in range(2):
        a = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in ring.primes]) for _ in range(batch)])
        b = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in ring.primes]) for _ in range(batch)])
        ta, tb = to_device(a), to_device(b)
        ref = _run(cuda, "vfhe_cuda_ntt_mul_intt_batch", ring, ta, tb)
        got = _run(cuda, "vfhe_cuda_ntt_mul_intt_batch_noalloc", ring, ta, tb)
        assert np.array_equal(got, ref)


def test_noalloc_rejects_oversized_batches(cuda):
    import torch

    from vfhe_b200.arith import Ring

    ring = Ring(2**16, prime_size=[50] * 4, split_degree=1, engine=cuda)
    batch = 5  # 5 * 4 * 2^16 residues > 2^20
    a = torch.zeros((batch, 4, 2**16), dtype=torch.int64, device="cuda")
    ffi = cuda.ffi
    limbs = ffi.new("uint32_t[]", ring.prime_indices)
    p = ffi.cast("uint64_t*", a.data_ptr())
    rc = cuda.lib.vfhe_cuda_ntt_mul_intt_batch_noalloc(ring.NTT, p, p, p, batch, limbs, 4, ffi.NULL)
    assert rc != 0
    assert "static scratch" in ffi.string(cuda.lib.vfhe_cuda_last_error()).decode()
    cuda.lib.vfhe_cuda_clear_error()


def test_noalloc_call_captures_into_a_cuda_graph(cuda):
    """The property the entry point exists for: after one warm call, a call captured by
    stream capture (global mode, where a cudaMalloc, cudaFree or synchronisation
    invalidates the capture) records and replays, and the replay's output equals the
    allocating entry's."""
    import torch

    from vfhe_b200.arith import Ring
    from vfhe_b200.batch import to_device

    N, batch = 4096, 16
    ring = Ring(N, prime_size=[50, 50, 50], split_degree=None, engine=cuda)
    rng = np.random.default_rng(5)
    a = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in ring.primes]) for _ in range(batch)])
    b = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in ring.primes]) for _ in range(batch)])
    ta, tb = to_device(a), to_device(b)
    ref = _run(cuda, "vfhe_cuda_ntt_mul_intt_batch", ring, ta, tb)
    _run(cuda, "vfhe_cuda_ntt_mul_intt_batch_noalloc", ring, ta, tb)  # warm: kernel attributes, scratch address

    ffi = cuda.ffi
    out = torch.zeros_like(ta)
    limbs = ffi.new("uint32_t[]", ring.prime_indices)
    p = lambda t: ffi.cast("uint64_t*", t.data_ptr())  # noqa: E731
    g = torch.cuda.CUDAGraph()
    rcs = []
    with torch.cuda.graph(g):
        st = ffi.cast("void*", torch.cuda.current_stream().cuda_stream)
        rcs.append(cuda.lib.vfhe_cuda_ntt_mul_intt_batch_noalloc(ring.NTT, p(out), p(ta), p(tb), batch, limbs,
                                                                ring.ell, st))
    assert rcs == [0], ffi.string(cuda.lib.vfhe_cuda_last_error()).decode()
    torch.cuda.synchronize()
    assert not out.any()  # captured, not run
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), ref)
    del g
