"""The bench's own arm on a B200: the JSON line carries the contract's keys with
consistent values (a short run: 2 timed whole evolutions, no CPU baseline, no DIS), and the
fixed-Sobol workload line agrees with the reference's C++ values it is compared with."""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def _line(*args: str) -> dict:
    result = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True,
                            timeout=900, cwd=ROOT)
    assert result.returncode == 0, result.stderr[-3000:]
    lines = [line for line in result.stdout.splitlines() if line.strip()]
    assert len(lines) == 1
    return json.loads(lines[0])


def test_bench_line_contract():
    d = _line("--steps", "2", "--warmup", "3", "--e2e-steps", "1", "--no-cpu-baseline", "--no-dis", "--no-batch")
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "roofline", "clocks",
                "max_rel_err_vs_fp64", "accuracy"):
        assert key in d, key
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] == 3
    # a step is one whole evolution to Y = 10: value is its mean device time, not a scaled one
    assert d["value"] == pytest.approx(d["ms_per_step"] / 1000, rel=1e-3)
    lo, hi = d["step_ms_min_max"]
    assert lo <= d["ms_per_step"] <= hi
    assert d["gpu_launches"] == 28 * 100 * 2
    # the headline precision bound, against the all-FP64 device build on the same points
    assert 0 < d["max_rel_err_vs_fp64"] <= 1e-4
    assert d["accuracy"]["rows_compared"] == 100
    e2e = d["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    roof = d["roofline"]
    assert roof["bound"] == "fp32" and roof["unit"] == "TFLOP/s"
    assert 0 < roof["frac"] < 1.5 and roof["frac"] == pytest.approx(roof["achieved"] / roof["peak"], rel=1e-2)
    assert 0 < roof["transcendental"]["frac"] < 1.5
    assert roof["census"]["flops_per_eval"] > 0
    assert roof["traffic"] > 0


def test_fixed_sobol_workload_line():
    d = _line("--workload", "fixed")
    assert d["value"] > 0 and d["baseline"]["value"] > d["value"]
    assert d["speedup_vs_cpp"] == pytest.approx(d["baseline"]["value"] / d["value"], rel=1e-2)
    # the six terms agree with the reference's C++ values within 5 combined standard errors
    cpp = {"L_I1": (0.10206739088678346, 0.0002535000977528945),
           "L_I2": (-0.024439455902300525, 0.00004764427185133986),
           "L_I3": (0.009414936380564324, 0.000026852425497947778),
           "T_I1": (0.40263591173620866, 0.0017956984452001683),
           "T_I2": (-0.08719375357937224, 0.00026850014906050766),
           "T_I3": (0.04848797141670969, 0.00013338145018266037)}
    for name, (ref, ref_err) in cpp.items():
        value, err = d["terms"][name]
        assert abs(value - ref) <= 5 * (err * err + ref_err * ref_err) ** 0.5, name


def test_batch_and_serve_lines():
    d = _line("--workload", "batch", "--batch-sets", "6")
    assert d["config"]["sets"] == 6 and d["config"]["points"] == 48
    assert d["value"] > 0 and d["batched_s"] > 0
    assert d["speedup_vs_plain_single_point"] > 0 and d["speedup_vs_plain_per_set"] > 0
    assert d["single_vs_batched_max_rel"] <= 1e-6
    s = _line("--workload", "serve", "--serve-seconds", "0.05", "--serve-rate", "100")
    assert s["value"] > 0 and s["p99_s"] >= s["p50_s"] > 0
    assert s["dis_batches"] >= 1 and s["speedup_vs_sequential"] > 0
