"""Serving loop (vfhe_cuda_server_*): every request's result is the same alone (plain
one-request-per-call server) and in a continuously batched mix, and equals the direct
batched entry points; the HBM budget is enforced."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mix(cuda, kind="rns"):
    from vfhe_b200.serve import ServingMix

    cggi = (256, 16) if kind == "rns" else (512, 32)
    return ServingMix(cuda, ckks=((2**12, 4), (2**13, 5)), cggi=cggi, cggi_max=16, pool=2, gens=2, seed=3,
                      cggi_kind=kind)


@pytest.mark.parametrize("kind", ["rns", "torus"])
def test_results_identical_alone_and_in_mix(cuda, kind):
    import torch

    from vfhe_b200.serve import Server, poisson_arrivals, run_stream

    mix = _mix(cuda, kind)
    reqs = mix.requests(48, seed=1, ckks_share=0.75, cggi_counts=(1, 16))
    assert {r[0] for r in reqs} == {"mul", "rot", "cggi"}

    plain = Server(8 << 30, streams=1, max_batch=1, engine=cuda)
    mix.register(plain)
    alone = run_stream(mix, plain, reqs, np.zeros(len(reqs)), keep_outputs=True)
    st_plain = plain.stats()
    plain.close()

    served = Server(8 << 30, streams=3, max_batch=8, engine=cuda)
    mix.register(served)
    arrivals = poisson_arrivals(20000.0, len(reqs), np.random.default_rng(2))
    mixed = run_stream(mix, served, reqs, arrivals, keep_outputs=True)
    st = served.stats()
    served.close()

    assert st_plain["batches"] == len(reqs) and st_plain["failed"] == 0
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["batches"] < len(reqs)  # requests were batched together
    for r, a, b in zip(reqs, alone["outputs"], mixed["outputs"]):
        for x, y in zip(a, b):
            assert torch.equal(x, y), r
    assert mixed["p99_ms"] >= mixed["p50_ms"] > 0


def test_served_results_equal_direct_batched_calls(cuda):
    import torch

    from vfhe_b200.batch import CkksBatch
    from vfhe_b200.serve import Server, run_stream

    mix = _mix(cuda)
    reqs = [r for r in mix.requests(30, seed=4, cggi_counts=(1, 16))]
    srv = Server(8 << 30, streams=2, max_batch=4, engine=cuda)
    mix.register(srv)
    res = run_stream(mix, srv, reqs, np.zeros(len(reqs)), keep_outputs=True)
    srv.close()
    ffi, lib = cuda.ffi, cuda.lib
    for r, outs in zip(reqs, res["outputs"]):
        kind, pi, x, y = r
        if kind == "mul":
            p = mix.ckks[pi]
            want = CkksBatch(p.ring[1], p.special, cuda).mul_relin_rescale(p.cts[x][None], p.cts[y][None], p.rlk)[0]
        elif kind == "rot":
            p = mix.ckks[pi]
            want = CkksBatch(p.ring[2], p.special, cuda).rotate(p.rcts[x][None], [y], [p.gks[y]])[0]
        else:
            cg = mix.cggi
            oa = torch.empty((x, 2, cg.N), dtype=torch.int64, device="cuda")
            ob = torch.empty((x, 2), dtype=torch.int64, device="cuda")
            limbs = ffi.new("uint32_t[]", list(cg.ring.prime_indices))
            ws = torch.empty(lib.vfhe_cuda_cggi_workspace_bytes(cg.ring.NTT, x, cg.n, 2) // 8 + 1,
                             dtype=torch.int64, device="cuda")
            P = lambda t: ffi.cast("uint64_t*", t.data_ptr())  # noqa: E731
            assert lib.vfhe_cuda_cggi_bootstrap_batch(
                cg.ring.NTT, P(oa), P(ob), P(cg.a[y:y + x].contiguous()), P(cg.b[y:y + x].contiguous()), x, cg.n,
                limbs, 2, cg.special, P(cg.bk), P(cg.tv), 16, ffi.cast("void*", ws.data_ptr()),
                ffi.cast("void*", torch.cuda.current_stream().cuda_stream)) == 0
            torch.cuda.synchronize()
            assert torch.equal(outs[0], oa) and torch.equal(outs[1], ob), r
            continue
        torch.cuda.synchronize()
        assert torch.equal(outs[0], want), r


def test_budget_limits_admission(cuda):
    from vfhe_b200.native import EngineError
    from vfhe_b200.serve import Server, ServingMix, run_stream

    mix = ServingMix(cuda, ckks=((2**12, 4), (2**13, 5)), pool=2, gens=1, seed=5, with_cggi=False)
    small = [r for r in mix.requests(40, seed=6) if r[1] == 0][:6]
    big = [r for r in mix.requests(40, seed=7) if r[1] == 1 and r[0] == "mul"][:1]
    assert small and big
    # room for the resident data and one small request's scratch, not for a level-5 multiply
    one_small = 8 * (4 * 4 * 2**12 + 2 * 3 * 2**12 + 2**12 * (3 * 4 + 4 * 5 + 2 * 5)) + (1 << 20)
    srv = Server(mix.resident + one_small, streams=2, max_batch=4, engine=cuda)
    mix.register(srv)
    res = run_stream(mix, srv, small, np.zeros(len(small)))
    assert res["requests"] == len(small)
    st = srv.stats()
    assert st["failed"] == 0 and st["batched_requests"] == len(small)
    out = mix.output_for(big[0])
    rid = mix.submit(srv, big[0], out)
    with pytest.raises(EngineError):
        srv.wait(rid)
    cuda.lib.vfhe_cuda_clear_error()
    srv.close()


def test_torus_requests_equal_direct_bootstraps_and_decrypt(cuda):
    """Torus CGGI requests served in a mix equal the direct programmable bootstrap of
    the same LWEs, and decrypt to the lookup table's values."""
    import torch

    from vfhe_b200.cggi_fft import to_host
    from vfhe_b200.serve import Server, run_stream

    mix = _mix(cuda, "torus")
    reqs = [r for r in mix.requests(30, seed=9, ckks_share=0.5, cggi_counts=(1, 16)) if r[0] == "cggi"]
    assert reqs
    srv = Server(8 << 30, streams=2, max_batch=4, engine=cuda)
    mix.register(srv)
    res = run_stream(mix, srv, reqs, np.zeros(len(reqs)), keep_outputs=True)
    srv.close()
    cg = mix.cggi
    for (kind, pi, x, y), outs in zip(reqs, res["outputs"]):
        want = cg.dev.bootstrap(cg.lwe[y:y + x], cg.tv)
        torch.cuda.synchronize()
        assert torch.equal(outs[0], want)
        assert np.array_equal(cg.keys.decrypt(to_host(outs[0])), cg.lut[cg.msgs[y:y + x]])
