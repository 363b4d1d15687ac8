"""Two-pass transforms as one dataflow launch (schedule ctas_per_sm = -2, ntt_flow.cu).

The launch interleaves the column pass and the tile pass of a split transform by
ticket; its results must equal the two-kernel schedule's bit for bit, forward and
inverse, for every supported (tile bits, column bits) pair, for row counts from one
row (every second-pass item waits on the first pass) to many (the interleave in its
steady state), for the digit broadcast (inputs reduced modulo another prime on load)
and for the CKKS pipeline.  Allocation-free callers and stream capture fall back to the
two kernels with the same results.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bucket(nrows: int) -> int:
    return nrows.bit_length() - 1


class _Schedule:
    """Set one (logP, bucket) schedule for the duration of a with-block."""

    def __init__(self, lib, ffi, logP, nrows, sched):
        self.lib, self.ffi, self.logP, self.nrows, self.sched = lib, ffi, logP, nrows, sched

    def __enter__(self):
        self.saved = self.ffi.new("int32_t[3]")
        self.lib.vfhe_cuda_ntt_get_schedule(self.logP, self.nrows, self.saved)
        assert self.lib.vfhe_cuda_ntt_set_schedule(self.logP, _bucket(self.nrows), *self.sched) == 0
        return self

    def __exit__(self, *exc):
        assert self.lib.vfhe_cuda_ntt_set_schedule(self.logP, _bucket(self.nrows), *self.saved) == 0


def _fwd_inv(cuda, ring, rows, stream=None):
    import torch

    from vfhe_b200.batch import to_device

    ffi, lib = cuda.ffi, cuda.lib
    st = ffi.cast("void*", (stream or torch.cuda.current_stream()).cuda_stream)
    B, L = rows.shape[0], rows.shape[1]
    limbs = ffi.new("uint32_t[]", ring.prime_indices[:L])
    x = to_device(rows)
    p = ffi.cast("uint64_t*", x.data_ptr())
    assert lib.vfhe_cuda_ntt_batch(ring.NTT, 0, p, p, B, limbs, L, st) == 0
    f = x.clone()
    assert lib.vfhe_cuda_ntt_batch(ring.NTT, 1, p, p, B, limbs, L, st) == 0
    torch.cuda.synchronize()
    return f.cpu().numpy().view(np.uint64), x.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("logP,K,B,per", [
    (13, 10, 3, 0), (13, 11, 1, 1), (14, 10, 1, 0), (14, 10, 40, 1), (14, 10, 40, 2), (14, 11, 7, 2),
    (14, 12, 2, 1), (15, 11, 5, 2), (15, 12, 1, 1), (15, 13, 2, 0), (16, 12, 1, 2), (16, 12, 24, 1),
    (16, 12, 24, 2), (16, 13, 3, 1), (17, 13, 2, 2),
])
def test_flow_schedule_matches_two_kernels(cuda, logP, K, B, per):
    from vfhe_b200.arith import Ring

    ffi, lib = cuda.ffi, cuda.lib
    N = 1 << logP
    ring = Ring(N, prime_size=[50, 49, 40], split_degree=1, engine=cuda)
    rng = np.random.default_rng(logP * 100 + K * 10 + B)
    rows = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in ring.primes]) for _ in range(B)])
    # canonical extremes in the first row
    rows[0, :, :4] = 0
    rows[0, :, 4:8] = np.array(ring.primes, dtype=np.uint64)[:, None] - 1
    nrows = B * 3
    with _Schedule(lib, ffi, logP, nrows, (K, 0, 0)):
        base_f, base_i = _fwd_inv(cuda, ring, rows)
    assert np.array_equal(base_i, rows)
    with _Schedule(lib, ffi, logP, nrows, (K, per, -2)):  # per: work items per ticket (0: two)
        got = ffi.new("int32_t[3]")
        lib.vfhe_cuda_ntt_get_schedule(logP, nrows, got)
        assert list(got) == [K, per, -2]
        launches0 = lib.vfhe_cuda_launch_count()
        f, i = _fwd_inv(cuda, ring, rows)
        assert lib.vfhe_cuda_launch_count() - launches0 == 2  # one launch per transform
    assert np.array_equal(f, base_f), (logP, K, B, per)
    assert np.array_equal(i, rows), (logP, K, B, per)
    assert lib.vfhe_cuda_device_faults() == 0


def test_flow_matches_oracle(cuda, oracle_engine):
    """Forward and inverse transforms of one polynomial through the reference API
    (Polynomial.to_NTT / to_coeff) on the cuda engine under the dataflow schedule and on
    the oracle engine."""
    from tests.helpers import poly_from_rows, same, twin_rings, uniform_rows

    ffi, lib = cuda.ffi, cuda.lib
    N = 2**14
    rg, ro = twin_rings([cuda, oracle_engine], N, [50, 50, 45, 40], split=1)
    rows = uniform_rows(rg, np.random.default_rng(11))
    pg, po = poly_from_rows(rg, rows), poly_from_rows(ro, rows)
    with _Schedule(lib, ffi, 14, 4, (10, 0, -2)):
        pg.to_NTT()
        po.to_NTT()
        same(pg, po)
        pg.to_coeff()
        po.to_coeff()
        same(pg, po)
    assert np.array_equal(pg.rows(), rows)
    assert lib.vfhe_cuda_device_faults() == 0


def test_flow_key_switch_digits_and_ckks_batch(cuda):
    """The batched CKKS multiply + rotation at N = 2^14, L = 9 + 1 (its key-switch digit
    transforms reduce their inputs modulo each extended prime on load) under the
    dataflow schedule for every row-count class equals the two-kernel schedules."""
    import torch

    from tests.test_gpu_batch import _setup
    from vfhe_b200.batch import CkksBatch, ciphertext_rows, key_tensor, to_device, to_host

    ffi, lib = cuda.ffi, cuda.lib
    N, steps = 2**14, [1, 4]
    s, key, rlk, gks, cts = _setup(cuda, N, 8, 16, steps, seed=41)
    for c in cts:
        c.to_NTT()
    t1 = to_device(np.stack([ciphertext_rows(c) for c in cts[0::2]]))
    t2 = to_device(np.stack([ciphertext_rows(c) for c in cts[1::2]]))
    special = s.special_rings[0].prime_indices[-1]
    gens = [s.galois_gen(steps[i % 2]) for i in range(8)]
    keys = {k: key_tensor(v) for k, v in gks.items()}
    kl = [keys[steps[i % 2]] for i in range(8)]

    def run():
        out = CkksBatch(s.rings[0], special).mul_relin_rescale(t1, t2, key_tensor(rlk))
        rot = CkksBatch(s.rings[1], special).rotate(out, gens, kl)
        torch.cuda.synchronize()
        return to_host(out), to_host(rot)

    base = run()
    saved = []
    for b in range(0, 16):  # every row-count class of 2^14-point transforms in this run
        sv = ffi.new("int32_t[3]")
        lib.vfhe_cuda_ntt_get_schedule(14, 1 << b, sv)
        saved.append((b, list(sv)))
        assert lib.vfhe_cuda_ntt_set_schedule(14, b, 10, 0, -2) == 0
    try:
        got = run()
    finally:
        for b, sv in saved:
            assert lib.vfhe_cuda_ntt_set_schedule(14, b, *sv) == 0
    assert np.array_equal(base[0], got[0])
    assert np.array_equal(base[1], got[1])
    assert lib.vfhe_cuda_device_faults() == 0


def test_flow_falls_back_without_allocation(cuda):
    """On a stream without a counter buffer, the allocation-free entry point takes the
    two-kernel path; the results are those of the allocating entry point."""
    import torch

    from vfhe_b200.arith import Ring
    from vfhe_b200.batch import to_device

    ffi, lib = cuda.ffi, cuda.lib
    N, B = 2**14, 2
    ring = Ring(N, prime_size=[50] * 3, split_degree=1, engine=cuda)
    rng = np.random.default_rng(3)
    a = to_device(np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in ring.primes]) for _ in range(B)]))
    b = to_device(np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in ring.primes]) for _ in range(B)]))
    limbs = ffi.new("uint32_t[]", ring.prime_indices)
    p = lambda t: ffi.cast("uint64_t*", t.data_ptr())  # noqa: E731
    outs = []
    torch.cuda.synchronize()  # the inputs are complete before other streams read them
    with _Schedule(lib, ffi, 14, B * 3, (10, 0, -2)):
        for fn in ("vfhe_cuda_ntt_mul_intt_batch_noalloc", "vfhe_cuda_ntt_mul_intt_batch"):
            fresh = torch.cuda.Stream()  # no counter buffer yet on this stream
            out = torch.empty_like(a)
            st = ffi.cast("void*", fresh.cuda_stream)
            assert getattr(lib, fn)(ring.NTT, p(out), p(a), p(b), B, limbs, 3, st) == 0
            fresh.synchronize()
            outs.append(out.cpu())
    assert torch.equal(outs[0], outs[1])
    assert lib.vfhe_cuda_device_faults() == 0


def test_flow_under_stream_capture(cuda):
    """Captured into a CUDA graph, the dataflow schedule records the two kernels; the
    replay equals the direct call."""
    import torch

    from vfhe_b200.arith import Ring
    from vfhe_b200.batch import to_device

    ffi, lib = cuda.ffi, cuda.lib
    N, B = 2**16, 2
    ring = Ring(N, prime_size=[50] * 2, split_degree=1, engine=cuda)
    rng = np.random.default_rng(4)
    rows = np.stack([np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in ring.primes]) for _ in range(B)])
    limbs = ffi.new("uint32_t[]", ring.prime_indices)
    with _Schedule(lib, ffi, 16, B * 2, (12, 0, -2)):
        want, _ = _fwd_inv(cuda, ring, rows)
        x = to_device(rows)
        s = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            st = ffi.cast("void*", s.cuda_stream)
            rc = lib.vfhe_cuda_ntt_batch(ring.NTT, 0, ffi.cast("uint64_t*", x.data_ptr()),
                                         ffi.cast("uint64_t*", x.data_ptr()), B, limbs, 2, st)
        assert rc == 0
        x.copy_(to_device(rows))
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(x.cpu().numpy().view(np.uint64), want)
        del g
    assert lib.vfhe_cuda_device_faults() == 0
