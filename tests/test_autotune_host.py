"""Autotuner host logic: candidate schedules are valid, tables apply to every bucket."""

from __future__ import annotations

import json


def test_candidates_respect_kernel_limits():
    from vfhe_b200.autotune import candidates

    for logP in range(8, 18):
        cands = candidates(logP)
        assert cands, logP
        assert (logP if logP <= 13 else 12, 0, 0) in cands  # the built-in schedule is always timed
        for k, tpc, cps in cands:
            assert 8 <= k <= 13 and k <= logP and logP - k <= 5
            assert tpc in (0, 1, 2, 4, 8) and cps in (0, 2, 4, -1, -2)
            if cps == -1:
                assert 11 <= k <= 13 and 1 <= logP - k <= 3
            if cps == -2:  # dataflow launch: 10..13 tile bits, radix 4..16 columns, one row per item
                assert 10 <= k <= 13 and 2 <= logP - k <= 4 and tpc in (1, 2)
                assert (max(256, 1 << (k - 4)) >> (k - 4)) <= (1 << (logP - k))
            if tpc and cps != -2:  # tiles one CTA holds (for -2: work items per ticket)
                assert (1 << (k - 4)) * tpc <= max(256, 1 << (k - 4))


class _FakeLib:
    def __init__(self):
        self.calls = []

    def vfhe_cuda_ntt_set_schedule(self, lp, b, tb, tpc, cps):
        self.calls.append((lp, b, tb, tpc, cps))
        return 0

    def vfhe_cuda_clear_error(self):
        pass


class _FakeEngine:
    def __init__(self):
        self.lib = _FakeLib()


def test_apply_fills_every_bucket_with_the_nearest_entry(tmp_path):
    from vfhe_b200 import autotune

    table = {"14/7": {"schedule": [13, 0, 0]}, "14/13": {"schedule": [12, 1, 2]}, "10/9": {"schedule": [10, 2, 0]}}
    eng = _FakeEngine()
    assert autotune.apply(eng, table) == 64
    got = {(lp, b): (tb, tpc, cps) for lp, b, tb, tpc, cps in eng.lib.calls}
    assert got[(14, 0)] == (13, 0, 0) and got[(14, 10)] == (13, 0, 0)  # ties go to the smaller bucket
    assert got[(14, 11)] == (12, 1, 2) and got[(14, 31)] == (12, 1, 2)
    assert all(got[(10, b)] == (10, 2, 0) for b in range(32))

    p = tmp_path / "t.json"
    p.write_text(json.dumps({"table": table}))
    assert autotune.load(p) == table
    assert autotune.load(tmp_path / "missing.json") is None


def test_dataflow_candidates_cover_the_two_pass_sizes():
    from vfhe_b200.autotune import candidates

    flows = {logP: sorted({k for k, _, cps in candidates(logP) if cps == -2}) for logP in range(8, 18)}
    assert flows[12] == [10] and flows[13] == [10, 11] and flows[14] == [10, 11, 12]
    assert flows[16] == [12, 13] and flows[17] == [13]
    assert all(not flows[lp] for lp in range(8, 12))

