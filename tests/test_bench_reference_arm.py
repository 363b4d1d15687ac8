"""bench.py --impl reference on the host: the CPU implementation of the path (the
reference's own library compiled from its sources, else the oracle port) timed on every
host core prints one JSON line with the same metric, unit and direction as the GPU arm,
an e2e equal to its value with no host-device bytes, and a cpu_baseline describing the
run; ranks other than 0 exit without work or output."""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(env_extra: dict) -> subprocess.CompletedProcess:
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_line():
    r = _run({})
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "CKKS mul+relin+rescale/s" and line["unit"] == "pairs/s"
    assert line["higher_is_better"] is True and line["scaling"] == "weak"
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert cb["sample"]
    assert line["config"]["N"] == 2**14 and line["config"]["L"] == 9


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
