"""bench.py's reference arm (the reference's algorithm timed on the host cores):
one JSON line with the contract's keys, on a tiny sample; ranks other than 0
exit quietly.  No device."""

from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
        "cpu_baseline", "e2e"}


def _run(args, env_extra=None):
    env = dict(os.environ, **(env_extra or {}))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl",
                           "reference", "--steps", "1", "--warmup", "0", "--cpu-seconds", "0.2",
                           *args], capture_output=True, text=True, timeout=240, env=env,
                          cwd=ROOT)


@pytest.mark.parametrize("args", [["--curves", "16", "--ref-curves", "2"], ["--workload", "tls", "--tls-curves", "2"],
                                  ["--workload", "multiband-shared", "--stars", "2"]])
def test_reference_arm_prints_one_contract_line(args):
    res = _run(args)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert KEYS <= set(out), KEYS - set(out)
    assert out["impl"] == "reference" and out["value"] > 0.0
    assert out["e2e"]["value"] == out["value"]
    assert out["e2e"]["h2d_bytes_per_step"] == 0 == out["e2e"]["d2h_bytes_per_step"]
    assert {"value", "unit", "cores", "kind", "sample"} <= set(out["cpu_baseline"])
    assert out["cpu_baseline"]["kind"] == "port"


def test_reference_arm_runs_on_rank_0_only():
    res = _run(["--curves", "16", "--ref-curves", "2"], {"RANK": "1", "WORLD_SIZE": "2"})
    assert res.returncode == 0, res.stderr[-2000:]
    assert not [l for l in res.stdout.splitlines() if l.startswith("{")]
