"""Time the reference's own BK evolution on the CPU, as shipped -- measurement infrastructure.

The reference package (torch_nlo_clean/src/nlo_torch) cannot travel to the GPU machine, so
its own CPU path is timed here, once, and the result is committed beside this script as
``reference_cpu_timing.json``; ``bench.py`` reports it as a secondary baseline with this
provenance.  What runs is the reference's public call
``solve_bk(MV(qs0sqr=0.2), 0.4, BKConfig(), device="cpu", dtype=torch.float64, seed=0)``:
its defaults (RPOINTS = 100 on [1e-6, 30], MCINTPOINTS = 1e5, step 0.2), which on the CPU mean
adaptive Gauss-Kronrod K1, Vegas K2+Kf per parent and the adaptive RK2 stepper
(bk/evolution.py:33-58, 239-326, 354-488).  Its derivative count and the time per derivative
are recorded too.

    NLO_REFERENCE_ROOT=<checkout> python -m oracle.reference_cpu_timing [<checkout>] 2> progress.log

The run prints one progress line per derivative on stderr.  A run stopped before it reaches
Y = 0.4 (the adaptive stepper may keep rejecting steps, since the Vegas estimates of K2+Kf
carry noise at the stepper's tolerance) is recorded from that log instead, marked incomplete:

    python -m oracle.reference_cpu_timing --partial progress.log --stopped-after SECONDS
"""

from __future__ import annotations

import json
import os
import platform
import re
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUTPUT = HERE / "reference_cpu_timing.json"


def _cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


PROGRESS = re.compile(r"^derivative (\d+) done at ([0-9.]+) s$")


def partial_record(log_text: str, stopped_after: float, threads: int, torch_version: str) -> dict:
    """The record of a run stopped after `stopped_after` seconds, from its progress lines."""
    done = [(int(m.group(1)), float(m.group(2))) for m in map(PROGRESS.match, log_text.splitlines()) if m]
    if not done:
        raise ValueError("no progress lines in the log")
    n, last = done[-1]
    if stopped_after < last:
        raise ValueError("the run cannot stop before its last progress line")
    return {
        "call": "nlo_torch.solve_bk(MV(qs0sqr=0.2), 0.4, BKConfig(), device='cpu', dtype=torch.float64, seed=0)",
        "config": {"RPOINTS": 100, "MINR": 1e-6, "MAXR": 30.0, "MCINTPOINTS": 100000, "DE_SOLVER_STEP": 0.2,
                   "INTMETHOD_NLO": "VEGAS"},
        "completed": False,
        "seconds_to_y_0_4": None,
        "stopped_after_s": round(stopped_after, 1),
        "derivatives": n,
        "seconds_per_derivative": round(last / n, 2),
        "threads": threads,
        "cpu_model": _cpu_model(),
        "torch": torch_version,
        "where": "the build container (the reference package does not travel to the GPU machine)",
        "note": f"stopped after {stopped_after:.0f} s without reaching Y = 0.4; {n} derivatives evaluated",
    }


def main() -> None:
    if "--partial" in sys.argv:
        import torch

        log = Path(sys.argv[sys.argv.index("--partial") + 1])
        stopped = float(sys.argv[sys.argv.index("--stopped-after") + 1])
        result = partial_record(log.read_text(), stopped, torch.get_num_threads(), torch.__version__)
        OUTPUT.write_text(json.dumps(result, indent=1) + "\n")
        print(json.dumps(result))
        return
    root = next((a for a in sys.argv[1:] if Path(a).is_dir()), os.environ.get("NLO_REFERENCE_ROOT"))
    if not root:
        raise SystemExit("set NLO_REFERENCE_ROOT (or pass the checkout) to the reference checkout's root")
    sys.path.insert(0, str(Path(root) / "torch_nlo_clean" / "src"))
    import torch

    import nlo_torch.bk.evolution as evolution
    from nlo_torch.bk.config import BKConfig
    from nlo_torch.bk.initial_conditions import MV

    calls = {"n": 0}
    original = evolution._evolve_derivative

    def counted(*args, **kwargs):
        out = original(*args, **kwargs)
        calls["n"] += 1
        # progress on stderr: a run stopped early still gives the time per derivative
        print(f"derivative {calls['n']} done at {time.perf_counter() - t0:.1f} s", file=sys.stderr, flush=True)
        return out

    evolution._evolve_derivative = counted
    config = BKConfig()
    t0 = time.perf_counter()
    table = evolution.solve_bk(MV(qs0sqr=0.2), 0.4, config, device="cpu", dtype=torch.float64, seed=0)
    seconds = time.perf_counter() - t0
    result = {
        "call": "nlo_torch.solve_bk(MV(qs0sqr=0.2), 0.4, BKConfig(), device='cpu', dtype=torch.float64, seed=0)",
        "config": {"RPOINTS": config.RPOINTS, "MINR": config.MINR, "MAXR": config.MAXR,
                   "MCINTPOINTS": config.MCINTPOINTS, "DE_SOLVER_STEP": config.DE_SOLVER_STEP,
                   "INTMETHOD_NLO": config.INTMETHOD_NLO.name},
        "completed": True,
        "seconds_to_y_0_4": round(seconds, 2),
        "derivatives": calls["n"],
        "seconds_per_derivative": round(seconds / max(calls["n"], 1), 2),
        "rows": int(table.N.shape[0]),
        "threads": torch.get_num_threads(),
        "cpu_model": _cpu_model(),
        "torch": torch.__version__,
        "where": "the build container (the reference package does not travel to the GPU machine)",
    }
    OUTPUT.write_text(json.dumps(result, indent=1) + "\n")
    print(json.dumps(result))


if __name__ == "__main__":
    main()
