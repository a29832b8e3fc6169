"""The bench's reference arm on the host: one JSON line with the contract's keys, the
oracle timed on a bounded sample; ranks other than 0 exit without work."""

from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _run(extra_env: dict[str, str] | None = None) -> subprocess.CompletedProcess:
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                          capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)


def test_reference_arm_prints_the_contract_line():
    result = _run()
    assert result.returncode == 0, result.stderr[-2000:]
    lines = [line for line in result.stdout.splitlines() if line.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["higher_is_better"] is False and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("full NLO BK evolution")


def test_reference_arm_other_ranks_exit_silently():
    result = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert result.returncode == 0, result.stderr[-2000:]
    assert result.stdout.strip() == ""


def test_reference_cpu_timing_partial_record():
    """A reference CPU run stopped before Y = 0.4 is recorded from its progress lines,
    marked incomplete, with the time per derivative of the lines it printed."""
    from oracle.reference_cpu_timing import partial_record

    log = "\n".join(["starting", "derivative 1 done at 500.0 s", "derivative 2 done at 1010.0 s",
                     "derivative 3 done at 1530.0 s"])
    rec = partial_record(log, 1800.0, 8, "x")
    assert rec["completed"] is False and rec["seconds_to_y_0_4"] is None
    assert rec["derivatives"] == 3 and rec["seconds_per_derivative"] == 510.0
    assert rec["stopped_after_s"] == 1800.0 and rec["threads"] == 8
    with pytest.raises(ValueError):
        partial_record("nothing here", 10.0, 8, "x")
    with pytest.raises(ValueError):
        partial_record(log, 1000.0, 8, "x")
