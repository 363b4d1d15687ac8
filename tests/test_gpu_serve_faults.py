"""Failure handling of the serving loop, with faults made on the host only.

A batch launch that fails, a scratch allocation that fails, and a batch whose completion
is never observed (until the batch deadline fails its requests) are injected through
vfhe_cuda_server_inject_fault; queued requests are cancelled and waits run into their
deadline while admission is paused.  In every case the failing requests report their
status, the server keeps running, and every other request's result equals the direct
batched call's.  No GPU fault, trap or hang is involved.
"""

from __future__ import annotations

import time

import pytest

pytestmark = pytest.mark.gpu


def _mix(cuda):
    from vfhe_b200.serve import ServingMix

    return ServingMix(cuda, ckks=((2**12, 4),), pool=4, gens=1, seed=11, with_cggi=False)


def _server(cuda, mix):
    # the server's worker is the only thread that launches engine work while it runs,
    # so every direct reference result is computed before the server starts
    from vfhe_b200.serve import Server

    srv = Server(8 << 30, streams=2, max_batch=4, engine=cuda)
    mix.register(srv)
    return srv


def _direct(cuda, mix, req):
    import torch

    from vfhe_b200.batch import CkksBatch

    kind, pi, x, y = req
    p = mix.ckks[pi]
    if kind == "mul":
        out = CkksBatch(p.ring[1], p.special, cuda).mul_relin_rescale(p.cts[x][None], p.cts[y][None], p.rlk)[0]
    else:
        out = CkksBatch(p.ring[2], p.special, cuda).rotate(p.rcts[x][None], [y], [p.gks[y]])[0]
    torch.cuda.synchronize()
    return out


def _mul_requests(mix, count, seed):
    return [r for r in mix.requests(4 * count, seed=seed) if r[0] == "mul"][:count]


def _submit_all(mix, srv, reqs):
    """Submit every request; returns the ids and the output tensors."""
    outs = [mix.output_for(r) for r in reqs]
    return [mix.submit(srv, r, o) for r, o in zip(reqs, outs)], outs


def test_failed_launch_fails_its_batch_only(cuda):
    import torch

    from vfhe_b200.native import EngineError

    mix = _mix(cuda)
    reqs = _mul_requests(mix, 6, seed=1)
    more = _mul_requests(mix, 3, seed=2)
    want = [_direct(cuda, mix, r) for r in reqs + more]
    srv = _server(cuda, mix)
    srv.pause(True)
    srv.inject_fault("launch", 1)
    ids, outs = _submit_all(mix, srv, reqs)
    srv.pause(False)
    failed = 0
    for rid, o, w in zip(ids, outs, want):
        try:
            srv.wait(rid, timeout_ms=60000)
        except EngineError:
            failed += 1
            continue
        assert torch.equal(o[0], w)
    cuda.lib.vfhe_cuda_clear_error()
    assert failed == 4  # the first batch (max_batch requests) failed, nothing else
    # the server keeps serving
    ids, outs = _submit_all(mix, srv, more)
    for rid, o, w in zip(ids, outs, want[len(reqs):]):
        srv.wait(rid, timeout_ms=60000)
        assert torch.equal(o[0], w)
    assert srv.fault_stats()["injected_pending"] == 0
    srv.close()


def test_failed_allocation_is_retried(cuda):
    import torch

    mix = _mix(cuda)
    reqs = _mul_requests(mix, 5, seed=3)
    want = [_direct(cuda, mix, r) for r in reqs]
    srv = _server(cuda, mix)
    srv.pause(True)
    srv.inject_fault("alloc", 1)
    ids, outs = _submit_all(mix, srv, reqs)
    srv.pause(False)
    for rid, o, w in zip(ids, outs, want):
        srv.wait(rid, timeout_ms=60000)  # none fails: the batch was re-queued
        assert torch.equal(o[0], w)
    fs = srv.fault_stats()
    assert fs["alloc_retries"] >= 1 and fs["injected_pending"] == 0
    assert srv.stats()["failed"] == 0
    srv.close()


def test_batch_deadline_fails_unobserved_batch(cuda):
    import torch

    from vfhe_b200.native import EngineError

    mix = _mix(cuda)
    reqs = _mul_requests(mix, 4, seed=4)
    more = _mul_requests(mix, 4, seed=5)
    want = [_direct(cuda, mix, r) for r in more]
    srv = _server(cuda, mix)
    srv.set_batch_timeout(300.0)
    srv.pause(True)
    srv.inject_fault("stall", 1)
    ids, outs = _submit_all(mix, srv, reqs)
    t0 = time.monotonic()
    srv.pause(False)
    for rid in ids:
        with pytest.raises(EngineError):
            srv.wait(rid, timeout_ms=60000)
    elapsed = time.monotonic() - t0
    assert 0.25 < elapsed < 30.0
    cuda.lib.vfhe_cuda_clear_error()
    assert srv.fault_stats()["expired_batches"] == 1
    # later batches complete normally (the stalled batch's stream was released)
    ids, outs = _submit_all(mix, srv, more)
    for rid, o, w in zip(ids, outs, want):
        srv.wait(rid, timeout_ms=60000)
        assert torch.equal(o[0], w)
    srv.close()


def test_cancel_and_wait_deadline(cuda):
    import torch

    from vfhe_b200.native import EngineError

    mix = _mix(cuda)
    reqs = _mul_requests(mix, 3, seed=6)
    want = [_direct(cuda, mix, r) for r in reqs]
    srv = _server(cuda, mix)
    srv.pause(True)
    ids, outs = _submit_all(mix, srv, reqs)
    with pytest.raises(TimeoutError):  # admission is held: the wait runs out, the request stays
        srv.wait(ids[0], timeout_ms=50)
    assert srv.poll(ids[1], timeout_ms=0) == 2
    assert srv.cancel(ids[1])
    assert srv.cancel(ids[1]) is False  # already finished (cancelled)
    srv.pause(False)
    for k in (0, 2):
        srv.wait(ids[k], timeout_ms=60000)
        assert torch.equal(outs[k][0], want[k])
    with pytest.raises(EngineError):
        srv.wait(ids[1])  # cancelled
    assert srv.fault_stats()["cancelled"] == 1
    assert srv.stats()["completed"] == 2
    srv.close()
