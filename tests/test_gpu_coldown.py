"""The key-switch accumulator's inverse column pass fused with the special-prime
division and the rescale (k_coldown, ckks.cu) must give the residues of the unfused
form (the whole inverse transform, then k_moddown) and of the one-op-per-call path.

The fused kernel runs where the 2^logP-point transform's schedule is a tile pass plus
a column pass of 2..16 points; the schedules are set here for every row-count class so
that each column width (1..4 bits) and the split layouts are exercised whatever the
tuned table says.  VFHE_CUDA_CKKS_UNFUSED=1 selects the unfused form in the same build.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from tests.test_gpu_batch import _setup

pytestmark = pytest.mark.gpu


class _AllBuckets:
    """Set the schedule of every row-count class of logP for the duration of a with-block."""

    def __init__(self, lib, ffi, logP, sched):
        self.lib, self.ffi, self.logP, self.sched = lib, ffi, logP, sched

    def __enter__(self):
        self.saved = []
        for b in range(32):
            sv = self.ffi.new("int32_t[3]")
            self.lib.vfhe_cuda_ntt_get_schedule(self.logP, 1 << b, sv)
            self.saved.append((b, list(sv)))
            assert self.lib.vfhe_cuda_ntt_set_schedule(self.logP, b, *self.sched) == 0
        return self

    def __exit__(self, *exc):
        for b, sv in self.saved:
            assert self.lib.vfhe_cuda_ntt_set_schedule(self.logP, b, *sv) == 0


def _run(cuda, s, rlk, gks, c1, c2, rot_steps, unfused: bool):
    import torch

    from vfhe_b200.batch import CkksBatch, ciphertext_rows, key_tensor, to_device, to_host

    t1 = to_device(np.stack([ciphertext_rows(c) for c in c1]))
    t2 = to_device(np.stack([ciphertext_rows(c) for c in c2]))
    special = s.special_rings[0].prime_indices[-1]
    keys = {k: key_tensor(v) for k, v in gks.items()}
    old = os.environ.get("VFHE_CUDA_CKKS_UNFUSED")
    os.environ["VFHE_CUDA_CKKS_UNFUSED"] = "1" if unfused else "0"
    try:
        n0 = cuda.lib.vfhe_cuda_launch_count()
        out = CkksBatch(s.rings[0], special).mul_relin_rescale(t1, t2, key_tensor(rlk))
        rot = CkksBatch(s.rings[1], special).rotate(out, [s.galois_gen(k) for k in rot_steps],
                                                    [keys[k] for k in rot_steps])
        torch.cuda.synchronize()
        launches = cuda.lib.vfhe_cuda_launch_count() - n0
    finally:
        if old is None:
            del os.environ["VFHE_CUDA_CKKS_UNFUSED"]
        else:
            os.environ["VFHE_CUDA_CKKS_UNFUSED"] = old
    cuda.check("coldown")
    return to_host(out), to_host(rot), launches


@pytest.mark.parametrize("N,n_mid,split,tile_bits", [
    (2**14, 8, 1, 10),   # the CKKS configuration's shape: radix-16 column pass
    (2**14, 8, 1, 11),   # radix 8
    (2**13, 4, 1, 11),   # radix 4
    (2**12, 3, 1, 11),   # radix 2
    (2**14, 3, 2, 10),   # split 2: two 2^13-point blocks per row, radix 8
    (2**12, 3, 4, 8),    # split 4 (the reference's default for these primes): 2^10-point blocks, radix 4
])
def test_fused_column_division_matches_unfused_and_single_calls(cuda, N, n_mid, split, tile_bits):
    from vfhe_b200.batch import ciphertext_rows

    steps = [1, 4]
    s, key, rlk, gks, cts = _setup(cuda, N, n_mid, 6, steps, seed=57, split=split)
    c1, c2 = cts[0::2], cts[1::2]
    rot_steps = [steps[i % len(steps)] for i in range(len(c1))]
    ref_prod, ref_rot = [], []
    for a, b, k in zip(c1, c2, rot_steps):
        p = s.multiply(a, b, rlk)
        p.round_division(lvl=1)
        ref_prod.append(ciphertext_rows(p))
        ref_rot.append(ciphertext_rows(s.automorphism(p, s.galois_gen(k), gks[k])))
    for c in cts:
        c.to_NTT()
    logP = (N // split).bit_length() - 1
    with _AllBuckets(cuda.lib, cuda.ffi, logP, (tile_bits, 0, 0)):
        fused = _run(cuda, s, rlk, gks, c1, c2, rot_steps, unfused=False)
        plain = _run(cuda, s, rlk, gks, c1, c2, rot_steps, unfused=True)
    assert np.array_equal(fused[0], np.stack(ref_prod))
    assert np.array_equal(fused[1], np.stack(ref_rot))
    assert np.array_equal(plain[0], fused[0]) and np.array_equal(plain[1], fused[1])
    # the fused form replaces the column pass and the division of the multiply and of
    # the rotation with one kernel each
    assert plain[2] - fused[2] == 2
    assert cuda.lib.vfhe_cuda_device_faults() == 0
