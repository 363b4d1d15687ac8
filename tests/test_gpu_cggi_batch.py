"""Batched CGGI16 bootstrap (vfhe_cuda_cggi_bootstrap_batch) against the reference API
path (CGGI16.functional_bootstrap over mgsw_CMUX), bit for bit, and LUT correctness."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(cuda, N, n_lwe, count, seed, msg_prec=5):
    from vfhe_b200.arith import Ring
    from vfhe_b200.fhe import CGGI16
    from vfhe_b200.mlwe import LWE_Key, MLWE_Scheme, encrypt_lwe
    from vfhe_b200.native import use_engine

    with use_engine(cuda):
        rng = np.random.default_rng(seed)
        Rq = Ring(N, prime_size=[50, 50, 50], split_degree=1)
        in_ring = Rq.quotient_ring(ell=2)
        s = MLWE_Scheme(Rq, special_primes=1, module_rank=1, max_lvl=1)
        in_key_s = [int(v) for v in rng.integers(0, 2, n_lwe)]
        in_key = LWE_Key(ring=in_ring, key=in_key_s, n=n_lwe)
        out_key = s.key_gen_sparse(64, 3.2, ternary=False, rng=rng)
        cg = CGGI16(s)
        bk = cg.generate_bootstrap_key(in_key, out_key, rng=rng)
        t = 1 << (msg_prec - 1)
        lut = [int(v) for v in rng.integers(0, t, t)]
        tv = cg.LUT_packing(lut, t, msg_prec)
        msgs = [int(v) for v in rng.integers(0, t, count)]
        lwes = []
        for m in msgs:
            scaled = round(m * in_ring.q_l / (1 << msg_prec)) % in_ring.q_l
            lwes.append(encrypt_lwe(in_ring, in_key_s, [scaled % q for q in in_ring.primes], 3.2, rng))
        ok = out_key.extract_lwe_key()
        key2 = LWE_Key(ring=in_ring, key=ok.get_s(), n=ok.n)
        return s, cg, bk, tv, lwes, msgs, lut, t, in_ring, key2


@pytest.mark.parametrize("N,n_lwe,count", [(256, 16, 4), (1024, 64, 8)])
def test_batched_bootstrap_matches_reference_path(cuda, N, n_lwe, count):
    import torch

    from vfhe_b200.batch import CggiBatch, bootstrap_key_tensor, to_device, to_host
    from vfhe_b200.mlwe import LWE

    s, cg, bk, tv, lwes, msgs, lut, t, in_ring, key2 = _setup(cuda, N, n_lwe, count, seed=N + n_lwe)
    ref_a, ref_b = [], []
    for lwe in lwes:
        out = LWE(ring=in_ring)
        cg.functional_bootstrap(out, tv, lwe, bk, torus_base=t)
        ref_a.append(np.array(out.get_a(), dtype=np.uint64))
        ref_b.append(np.array(out.get_b(), dtype=np.uint64))

    a = to_device(np.stack([np.array(l.get_a(), dtype=np.uint64) for l in lwes]))
    b = to_device(np.stack([np.array(l.get_b(), dtype=np.uint64) for l in lwes]))
    tv.to_coeff()
    tvt = to_device(np.stack([tv.component_rows(0), tv.component_rows(1)]))
    oa, ob = CggiBatch(s).bootstrap(a, b, bootstrap_key_tensor(bk), tvt, t)
    torch.cuda.synchronize()
    assert np.array_equal(to_host(oa), np.stack(ref_a))
    assert np.array_equal(to_host(ob), np.stack(ref_b))

    # decryption of the batched outputs
    for i, m in enumerate(msgs):
        o = LWE(ring=in_ring, n=N)
        o.set_rows(to_host(oa)[i], to_host(ob)[i])
        ph = o.phase(key2, recompose=True)
        assert round(ph * (2 * t) / in_ring.q_l) % (2 * t) == lut[m]
