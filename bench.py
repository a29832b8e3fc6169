"""Benchmark: full NLO BK evolution to Y = 10 on B200.

Workload (the configuration the headline metric is quoted on): 400 log-spaced
parent sizes r in [1e-7, 1e2] GeV^-1, MV initial condition (Qs0^2 = 0.2 GeV^2,
gamma = 1, Lambda = 0.241 GeV), smooth-freeze Balitsky/smallest-dipole running
coupling, RK4 in rapidity with step 0.1 up to Y = 10, 2^20 scrambled Sobol points
per parent per stage for K2+Kf, the fixed 8 x 24 rule per r interval for K1;
FP32 integrands with FP64 sums, spline refit and RK update.

A bench "step" is one whole evolution from Y = 0 to Y = 10 (100 RK4 steps, 400
right-hand sides, one nlo_bk_evolve call); ``value`` is the mean device time of the K
timed evolutions, in seconds to Y = 10 -- measured, not scaled.  Outside the timed region
the same evolution runs once in the all-FP64 device build on the same Sobol points, and
``max_rel_err_vs_fp64`` is the largest relative difference of the timed build's rows.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (one process per GPU under torchrun) K2+Kf is sharded over the ranks
by Sobol index range and K1 by parent, with one NCCL all-reduce of dN/dY per RK stage;
the total work is fixed (strong scaling) and the value is the slowest rank's device time.

The line also carries a "dis" object: NLO DIS sigma_r throughput on a BK table evolved by
the same workload (see measure_dis); --workload dis prints that measurement alone.  And a
"fixed_sobol" object: the reference's own fixed-Sobol qqbar-g benchmark setting timed
against its published C++ time (see measure_fixed; --workload fixed alone).

--impl reference times the reference algorithm on the host cores (the oracle's
C restatement, all threads): each of its steps is one complete right-hand side of the
workload at a rapidity spread over 0..10 (amplitudes from the oracle's own evolution),
and the value is the mean stage time times the 400 stages.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "NLO BK s to Y=10 & DIS points/s at <=1e-4 rel err; served p50/p99 latency"
UNIT = "s to Y=10 (NLO BK evolution)"
MAXY = 10.0
STEP = 0.1
RPOINTS = 399
MINR, MAXR = 1e-7, 1e2
SAMPLES = 1 << 20
QS0SQR = 0.2
RK_STEPS = 100  # RK4 steps of one whole evolution (Y = 0 -> 10)
SAMPLES_LOG2 = 20
# Op census of one K2+Kf evaluation, from oracle/census.py (an op-counting run of the
# oracle's FP64 restatement of _nlo_integrand x Jacobian on the workload's points at the
# final state): per (sample, parent) pair, and per sample for the parent-independent part.
# Arithmetic = add, sub, mul, div, sqrt; transcendental = exp, log, sin, cos, expm1, log1p.
CENSUS_EVAL_FLOPS = 135
CENSUS_EVAL_TRANSCENDENTALS = 13
CENSUS_SAMPLE_FLOPS = 41
CENSUS_SAMPLE_TRANSCENDENTALS = 20
MUFU_PER_SM_PER_CLOCK = 16
# DRAM bytes of one K2+Kf launch (dram__bytes_read.sum + dram__bytes_write.sum) from the
# ncu capture of the kernel case (bench.py --kernel-case: 400 parents x 2^18 points): the
# spline is staged into shared memory once per CTA and each CTA writes 3 doubles per
# parent, so the bytes do not grow with the number of samples.
K2KF_DRAM_BYTES_PER_LAUNCH = 52224
# Launches of our kernels per RK4 step: 4 right-hand sides x (spline refit, active
# list, K1, K2+Kf, K2+Kf finalize, assemble) + 4 stage combinations.
LAUNCHES_PER_RK4_STEP = 4 * 6 + 4
SM_COUNT = 148
FP32_LANES_PER_SM = 128
# CPU baseline sample: complete right-hand sides spread over the evolution
CPU_STAGES = 3


def workload_config():
    from nlo_bk_optimized_b200 import BKConfig
    from nlo_bk_optimized_b200.bk.config import IntegrationMethod

    return BKConfig(RPOINTS=RPOINTS, MINR=MINR, MAXR=MAXR, MCINTPOINTS=SAMPLES, DE_SOLVER_STEP=STEP,
                    STEPPER="rk4", PRECISION="mixed", INTMETHOD_NLO=IntegrationMethod.SOBOL)


def workload_description(extra: dict | None = None) -> dict:
    out = {
        "workload": "full NLO BK evolution: 400 r in [1e-7,1e2] GeV^-1, MV Qs0^2=0.2, RK4 h=0.1 to Y=10, "
                    "2^20 scrambled Sobol points per r per stage, fixed 8x24 K1 rule",
        "r_points": RPOINTS + 1,
        "samples_per_r_per_stage": SAMPLES,
        "rk_step": STEP,
        "maxy": MAXY,
        "stepper": "rk4",
        "precision": "FP32 integrands, FP64 sums/spline/RK",
        "l2": "256 MiB buffer written between timed steps (working set is L2-resident by nature)",
    }
    if extra:
        out.update(extra)
    return out


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.file = None

    def __enter__(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        return False

    def summary(self) -> dict | None:
        if self.proc is None or self.file is None:
            return None
        self.file.flush()
        rows = []
        with open(self.file.name) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), float(parts[3]) if parts[3] not in ("", "[N/A]") else 0.0,
                                 parts[5], parts[6], parts[7], parts[8]))
                except ValueError:
                    continue
        os.unlink(self.file.name)
        if not rows:
            return None
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for row in rows:
            for name, flag in zip(names, row[3:]):
                if flag.lower() == "active":
                    reasons.add(name)
        loaded = [row[0] for row in rows]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(row[1] for row in rows),
                "power_w_max": max(row[2] for row in rows), "samples": len(rows), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    from nlo_bk_optimized_b200 import MV, _native, solve_bk
    from nlo_bk_optimized_b200.bk.evolution import _r_grid, nlo_box, params_of, workspace

    world, rank, local = dist_setup()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=device)

    config = workload_config()
    lib = _native.load()
    params = params_of(config, _native.PRECISION_MIXED)
    r_host = _r_grid(config, device="cpu", dtype=torch.float64)
    N0_host = MV(qs0sqr=QS0SQR).dipole_amplitude(r_host)
    r = r_host.to(device)
    points = r.numel()
    lower, width = nlo_box(float(r_host[0]), float(r_host[-1]))
    box = _native.box(lower, width)
    dirs = _native.sobol_dirs(4, 0)
    ws = workspace(device, points)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    stream = torch.cuda.current_stream(device)
    steps, warmup = args.steps, args.warmup
    table = torch.empty((RK_STEPS + 1, points), dtype=torch.float64, device=device)
    N0 = N0_host.to(device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)

    if world == 1:
        def evolution(precision_params) -> None:
            """One bench step: the whole evolution Y = 0 -> 10 (100 RK4 steps) in one call."""
            table[0].copy_(N0)
            _native.check(lib.nlo_bk_evolve(precision_params, r.data_ptr(), points, RK_STEPS, STEP,
                                            _native.STEPPERS["rk4"], dirs, SAMPLES, box, table.data_ptr(),
                                            status.data_ptr(), ws.data_ptr(), ws.numel(), stream.cuda_stream))
    else:
        # K2+Kf sharded over the ranks by Sobol index range, K1 by parent; one NCCL
        # all-reduce of the R-point derivative per stage (nlo_bk_optimized_b200/bk/sharded.py)
        from nlo_bk_optimized_b200.bk.sharded import ShardedRhs, shard_steps

        def evolution(precision_params) -> None:
            sharded = ShardedRhs(precision_params, r, dirs, SAMPLES, box, rank, world, ws, status, stream)
            table[0].copy_(N0)
            rows = shard_steps(table[0], RK_STEPS, STEP, "rk4", sharded.rhs,
                               lambda k: dist.all_reduce(k, op=dist.ReduceOp.SUM), sharded.stage, True)
            for i, row in enumerate(rows[1:], start=1):
                table[i].copy_(row)

    # warm-up: W whole evolutions (discarded)
    for _ in range(warmup):
        evolution(params)
    torch.cuda.synchronize()

    # timed region: K whole evolutions, the L2 flushed before each
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    with ClockSampler(local) as sampler:
        for i in range(steps):
            flush.zero_()
            starts[i].record(stream)
            evolution(params)
            ends[i].record(stream)
        torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    if world > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    if int(status.item()) != 0:
        raise FloatingPointError("non-finite amplitude in the benchmark evolution")
    clocks = sampler.summary()
    mixed_rows = table.clone()

    # accuracy of the timed (mixed) build: the same evolution on the same Sobol points in
    # the all-FP64 device build, outside the timed region
    params64 = params_of(config, _native.PRECISION_FP64)
    t64 = time.perf_counter()
    evolution(params64)
    torch.cuda.synchronize()
    fp64_s = time.perf_counter() - t64
    if int(status.item()) != 0:
        raise FloatingPointError("non-finite amplitude in the FP64 evolution")
    accuracy = mixed_vs_fp64(mixed_rows, table, r)
    final_N = mixed_rows[RK_STEPS].clone()

    # dominant kernel (K2+Kf) timed alone with events on its stream, at the final state
    idx = torch.empty(points, dtype=torch.int32, device=device)
    count = torch.empty(1, dtype=torch.int32, device=device)
    spline = torch.empty(int(lib.nlo_bk_spline_doubles(points)), dtype=torch.float64, device=device)
    _native.check(lib.nlo_bk_splines(r.data_ptr(), final_N.data_ptr(), points, 1, spline.data_ptr(), stream.cuda_stream))
    _native.check(lib.nlo_bk_active(final_N.data_ptr(), points, idx.data_ptr(), count.data_ptr(), stream.cuda_stream))
    k2_out = torch.empty((points, 3), dtype=torch.float64, device=device)
    k2_ws = torch.empty(int(lib.nlo_bk_k2kf_workspace_bytes(points)), dtype=torch.uint8, device=device)
    reps = 3
    k_start = [torch.cuda.Event(enable_timing=True) for _ in range(reps + 1)]
    k_end = [torch.cuda.Event(enable_timing=True) for _ in range(reps + 1)]
    for i in range(reps + 1):
        flush.zero_()
        k_start[i].record(stream)
        _native.check(lib.nlo_bk_k2kf(params, r.data_ptr(), points, spline.data_ptr(), idx.data_ptr(),
                                      count.data_ptr(), dirs, 0, SAMPLES, box, k2_out.data_ptr(), k2_ws.data_ptr(),
                                      k2_ws.numel(), stream.cuda_stream))
        k_end[i].record(stream)
    torch.cuda.synchronize()
    k2_ms = sum(k_start[i].elapsed_time(k_end[i]) for i in range(1, reps + 1)) / reps
    n_active = int(count.item())

    # end to end through the public API with host buffers, whole evolutions: the host
    # initial condition goes in, the full table comes back to the host
    if world == 1:
        def solve():
            return solve_bk(MV(qs0sqr=QS0SQR), MAXY, config, device=device, dtype=torch.float32, seed=0)
    else:
        from nlo_bk_optimized_b200.bk.sharded import solve_bk_sharded

        def solve():
            return solve_bk_sharded(MV(qs0sqr=QS0SQR), MAXY, config, device=device, dtype=torch.float32, seed=0)
    solve().N.cpu()  # one untimed call: the first call of a process pays one-time module loading
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e_reps = max(1, min(steps, args.e2e_steps))
    t0 = time.perf_counter()
    for _ in range(e2e_reps):
        host_table = solve().N.cpu()
    e2e_s = (time.perf_counter() - t0) / e2e_reps
    h2d = 2 * points * 8  # the r grid and the initial row (float64)
    d2h = host_table.numel() * host_table.element_size() + 4  # the table and the status word

    seconds = sum(step_ms) / steps / 1000.0
    if world > 1:
        t = torch.tensor([seconds, e2e_s], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        seconds, e2e_s = float(t[0]), float(t[1])
        dist.destroy_process_group()
    if rank != 0:
        return

    line = {
        "metric": METRIC,
        "value": round(seconds, 4),
        "unit": UNIT,
        "n_gpus": world,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": round(seconds * 1000.0, 3),
        "step": "one whole evolution Y = 0 -> 10 (100 RK4 steps, 400 right-hand sides)",
        "step_ms_min_max": [round(min(step_ms), 3), round(max(step_ms), 3)],
        "higher_is_better": False,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic (MV initial condition)",
        "config": workload_description({"parallelism": (f"K2+Kf Sobol range and K1 parents sharded over {world} "
                                                         "GPUs, one NCCL all-reduce of dN/dY per stage")
                                        if world > 1 else "single GPU",
                                        "active_parents_final": n_active}),
        "max_rel_err_vs_fp64": accuracy["max_rel_err"],
        "accuracy": dict(accuracy, fp64_evolution_s=round(fp64_s, 3),
                         reference="the all-FP64 device build of the same evolution on the same Sobol points"),
        "e2e": {"value": round(e2e_s, 4), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": e2e_reps,
                "api": ("nlo_bk_optimized_b200.solve_bk" if world == 1 else
                        "nlo_bk_optimized_b200.bk.sharded.solve_bk_sharded") + " + table.N.cpu()"},
        "gpu_launches": LAUNCHES_PER_RK4_STEP * RK_STEPS * steps,
        "roofline": k2kf_roofline(n_active, k2_ms),
        "clocks": clocks,
        "wall_s_timed_region": round(wall, 3),
    }
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline()
    timing = reference_torch_cpu()
    if timing is not None:
        line["reference_torch_cpu"] = timing
    if not args.no_dis and world == 1:
        # the second half of the metric: NLO DIS sigma_r points/s on an evolved table
        line["dis"] = measure_dis(args.dis_points, args.dis_single, args.dis_check)
        line["fixed_sobol"] = measure_fixed()
    if not args.no_batch and world == 1:
        line["batch"] = measure_batch(args.line_batch_sets)
        line["serve"] = measure_serve(args.line_serve_seconds, args.serve_rate, args.serve_slots, args.serve_waves)
    print(json.dumps(line))


def mixed_vs_fp64(mixed, fp64, r) -> dict:
    """Relative difference of the mixed build's rows from the FP64 build's, over every row
    after the initial one and every parent with N > 0 in the FP64 rows."""
    import torch

    m, f = mixed[1:].double(), fp64[1:].double()
    keep = f > 0
    rel = torch.where(keep, (m - f).abs() / f.abs().clamp_min(1e-300), torch.zeros_like(f))
    per_row = rel.max(dim=1).values
    per_parent = rel.max(dim=0).values
    worst = int(torch.argmax(per_parent))
    return {"max_rel_err": float(per_row.max()), "final_row_max_rel_err": float(per_row[-1]),
            "max_abs_err": float((m - f).abs().max()), "worst_parent_r": float(r[worst]),
            "rows_compared": int(f.shape[0]), "parents_compared": int(keep.any(dim=0).sum())}


def k2kf_roofline(n_active: int, k2_ms: float) -> dict:
    """Roofline of the dominant kernel from the op census of the FP64 restatement: per
    launch, every (sample, active parent) pair costs CENSUS_EVAL_FLOPS arithmetic operations
    and CENSUS_EVAL_TRANSCENDENTALS transcendental calls, and every sample costs
    CENSUS_SAMPLE_* once (the parent-independent part)."""
    evals = n_active * SAMPLES
    flops = evals * CENSUS_EVAL_FLOPS + SAMPLES * CENSUS_SAMPLE_FLOPS
    trans = evals * CENSUS_EVAL_TRANSCENDENTALS + SAMPLES * CENSUS_SAMPLE_TRANSCENDENTALS
    seconds = k2_ms * 1e-3
    sm_mhz = 1965.0
    peak = SM_COUNT * FP32_LANES_PER_SM * 2 * sm_mhz * 1e6 / 1e12
    mufu_peak = SM_COUNT * MUFU_PER_SM_PER_CLOCK * sm_mhz * 1e6
    achieved = flops / seconds / 1e12
    return {
        "bound": "fp32",
        "achieved": round(achieved, 3),
        "peak": round(peak, 2),
        "unit": "TFLOP/s",
        "frac": round(achieved / peak, 4),
        "traffic": K2KF_DRAM_BYTES_PER_LAUNCH,
        "kernel": "k2kf_kernel<float,true,0> (csrc/k2kf.cu)",
        "peak_source": "nominal FP32 (148 SM x 128 lanes x 2 x 1965 MHz); MEASURED_PEAKS.json has only HBM and bf16",
        "census": {"source": "oracle/census.py: op-counting run of the oracle's FP64 K2+Kf restatement",
                   "flops_per_eval": CENSUS_EVAL_FLOPS, "transcendentals_per_eval": CENSUS_EVAL_TRANSCENDENTALS,
                   "flops_per_sample": CENSUS_SAMPLE_FLOPS,
                   "transcendentals_per_sample": CENSUS_SAMPLE_TRANSCENDENTALS},
        "transcendental": {"achieved_per_s": round(trans / seconds, 1), "peak_per_s": mufu_peak,
                           "frac": round(trans / seconds / mufu_peak, 4),
                           "peak_source": "nominal 16 MUFU operations per SM per clock at 1965 MHz"},
        "evals_per_launch": evals,
        "launch_ms": round(k2_ms, 4),
        "evals_per_s": round(evals / seconds, 1),
        "traffic_source": "ncu capture of one K2+Kf launch (400 parents x 2^18 points); the spline is staged "
                          "once per CTA, so DRAM bytes do not grow with the sample count",
    }


# ---------------------------------------------------------------------------
def _rows_at(ys):
    """The oracle-evolved amplitude (oracle/evolution_rows_400r.npz) at rapidities ys,
    linear between the stored rows."""
    import numpy as np

    with np.load(ROOT / "oracle" / "evolution_rows_400r.npz") as data:
        r, y, N = data["r"], data["y"], data["N"]
    out = []
    for v in ys:
        k = int(min(max(np.searchsorted(y, v) - 1, 0), y.size - 2))
        t = (v - y[k]) / (y[k + 1] - y[k])
        out.append((1 - t) * N[k] + t * N[k + 1])
    return r, out


def _stage_seconds(N, r, points) -> tuple[float, int]:
    """Wall time of one complete right-hand side of the oracle (C, OpenMP, all host threads):
    the splines, K1 on every active parent, K2+Kf on every active parent x the given points."""
    import oracle

    phys = oracle.physics(workload_config())
    t0 = time.perf_counter()
    d = oracle.derivative(N, r, phys, points, True)
    return time.perf_counter() - t0, int((d.dNdy != 0).sum())


def _sobol_points():
    import oracle

    state, shift = oracle.sobol_state(4, 0)
    return oracle.sobol(state, shift, 0, SAMPLES, as_f32=True)


def _cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline() -> dict:
    """The oracle timed on a bounded sample of the workload: CPU_STAGES complete stages
    (2^20 points) spread over Y = 0..10, their mean times the 400 stages of the evolution."""
    import oracle

    ys = [MAXY * (k + 0.5) / CPU_STAGES for k in range(CPU_STAGES)]
    r, rows = _rows_at(ys)
    points = _sobol_points()
    times = [_stage_seconds(N, r, points)[0] for N in rows]
    mean = sum(times) / len(times)
    return {
        "value": round(mean * RK_STEPS * 4, 1),
        "unit": UNIT,
        "cores": oracle.num_threads(),
        "cpu_model": _cpu_model(),
        "kind": "port",
        "sample": (f"oracle (C, OpenMP): {CPU_STAGES} complete right-hand sides (every active parent, 2^20 Sobol "
                   f"points, K1 fixed rule) at Y = {', '.join(f'{v:.2f}' for v in ys)}, mean x 400 stages "
                   f"({sum(times):.1f} s measured)"),
        "measured_s": round(sum(times), 2),
        "extrapolation_factor": round(RK_STEPS * 4 / CPU_STAGES, 2),
    }


def reference_torch_cpu() -> dict | None:
    """The reference package's own CPU evolution as shipped (solve_bk(..., device="cpu",
    dtype=float64) at its defaults to Y = 0.4), timed once in the build container by
    oracle/reference_cpu_timing.py -- the package does not travel to the GPU machine.  A
    secondary baseline, reported with where it was measured; not used for any ratio."""
    path = ROOT / "oracle" / "reference_cpu_timing.json"
    if not path.exists():
        return None
    return json.loads(path.read_text())


def run_reference(args) -> None:
    """The reference algorithm on the host cores (the oracle's C restatement, all threads):
    each step is one complete right-hand side of the workload (splines, K1 on every active
    parent, K2+Kf on every active parent x 2^20 Sobol points), step i at rapidity
    Y_i = 10 (i + 1/2)/K on the oracle's own evolution rows; value = the mean stage time
    x the 400 stages of the evolution (only the stage count is extrapolated)."""
    world, rank, local = dist_setup()
    if rank != 0:
        return
    import oracle

    steps, warmup = args.steps, args.warmup
    ys = [MAXY * (k + 0.5) / steps for k in range(steps)]
    r, rows = _rows_at(ys)
    points = _sobol_points()
    for k in range(warmup):
        _stage_seconds(rows[k % len(rows)], r, points)
    t0 = time.perf_counter()
    times, active = [], []
    for N in rows:
        seconds, n_active = _stage_seconds(N, r, points)
        times.append(seconds)
        active.append(n_active)
    elapsed = time.perf_counter() - t0
    stage_s = sum(times) / steps
    seconds = stage_s * RK_STEPS * 4
    sample = (f"{steps} complete right-hand sides (every active parent, 2^20 Sobol points, K1 fixed rule) at "
              f"Y = {ys[0]:.2f}..{ys[-1]:.2f}; mean stage x 400 stages; {elapsed:.1f} s measured")
    line = {
        "metric": METRIC,
        "impl": "reference",
        "value": round(seconds, 2),
        "unit": UNIT,
        "n_gpus": world,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": round(stage_s * 1000, 2),
        "step": "one complete right-hand side (a quarter RK4 step) of the evolution",
        "higher_is_better": False,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (MV initial condition)",
        "config": workload_description({"parallelism": "host cores", "active_parents": active}),
        "measured_s": round(elapsed, 2),
        "extrapolation_factor": round(RK_STEPS * 4 / steps, 2),
        "cpu_baseline": {"value": round(seconds, 2), "unit": UNIT, "cores": oracle.num_threads(),
                         "cpu_model": _cpu_model(), "kind": "port", "sample": sample},
        "e2e": {"value": round(seconds, 2), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    timing = reference_torch_cpu()
    if timing is not None:
        line["reference_torch_cpu"] = timing
    print(json.dumps(line))


def run_kernel_case() -> None:
    """Small case for ncu captures: one K2+Kf launch (400 parents x 2^18 Sobol points)
    and one K1 launch at the initial condition, twice."""

    import torch

    from nlo_bk_optimized_b200 import MV, kernels
    from nlo_bk_optimized_b200.bk.evolution import _r_grid

    config = workload_config()
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    N = MV(qs0sqr=QS0SQR).dipole_amplitude(r)
    for _ in range(2):
        kernels.k2kf(r, N, config, samples=1 << 18)
        kernels.k1(r, N, config)
    torch.cuda.synchronize()
    print("kernel case done")


DIS_Q2 = (1.0, 50.0, 32)
DIS_X = (1e-5, 1e-2, 16)
DIS_SQRT_S = 318.0
DIS_SIGMA0_HALF_MB = 16.0
MB_TO_GEV2 = 2.56819
DIS_BINS, DIS_ITERATIONS, DIS_SAMPLES = 50, 10, 1 << 18


def run_dis_kernel_case() -> None:
    """Small DIS case for ncu captures: one (Q^2, x) point with the GBW dipole, one Vegas
    round of 2^16 Sobol points for each of the qqbar-g terms I1, I2 and I3 (nested, 48 inner
    nodes) in the mixed build, twice."""
    import torch

    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.dipole import GBW
    from nlo_bk_optimized_b200.dis import DISConfig, Polarization, Quark, QuarkType
    from nlo_bk_optimized_b200.dis.observables import kinematics
    from nlo_bk_optimized_b200.numerics.integration import VegasOptions, vegas_terms

    device = torch.device("cuda", 0)
    config = DISConfig(quarks=(Quark(QuarkType.LIGHT, 0.14),))
    kin = kinematics(10.0, 1e-3, Polarization.T, config, config.quarks[0])
    dip = GBW(Qs0sqr=0.25, lambda_=0.29, gamma=1.0, x0=0.01).native()
    opts = VegasOptions(samples_per_iteration=1 << 16, max_iterations=1, min_iterations=1, bins=DIS_BINS,
                        epsrel=1e-12)
    for _ in range(2):
        for term in ("I1", "I2N", "I3N"):
            vegas_terms(_native.DIS_TERMS[term], [kin], dip, opts, [0], precision=_native.PRECISION_MIXED,
                        device=device)
    torch.cuda.synchronize()
    print("dis kernel case done")


def measure_dis(points: int = 0, single: int = 4, check: int = 4) -> dict:
    """NLO DIS reduced cross section on an evolved BK table: 32 Q^2 log-spaced in [1, 50] GeV^2
    x 16 x_Bj log-spaced in [1e-5, 1e-2], sqrt(s) = 318 GeV, light quarks (m = 0.14 GeV,
    sum of charges^2 = 2/3), sigma_0/2 = 16 mb, Vegas 50 bins x 10 iterations x 2^18, seed 0.
    The table is the headline BK workload (400 r, 2^20 Sobol points, RK4 h = 0.1) evolved to
    Y = 16 (the qqbar-g terms reach Y = ln(Q^2/(x Q0^2)) = 15.4).  Timed: the batched
    structure_functions call over all points (value) and single-point sigma_r calls on a
    sample of points (the plain path)."""
    import torch

    from nlo_bk_optimized_b200 import MV, solve_bk
    from nlo_bk_optimized_b200.dipole import BKDipole
    from nlo_bk_optimized_b200.dis import DISConfig, DISOrder, Quark, QuarkType, sigma_r, structure_functions

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    config_bk = workload_config()
    table = solve_bk(MV(qs0sqr=QS0SQR), 16.0, config_bk, device=device, dtype=torch.float64, seed=0)
    dipole = BKDipole(table)
    Q2 = torch.logspace(math.log10(DIS_Q2[0]), math.log10(DIS_Q2[1]), DIS_Q2[2], dtype=torch.float64)
    xs = torch.logspace(math.log10(DIS_X[0]), math.log10(DIS_X[1]), DIS_X[2], dtype=torch.float64)
    Qg, Xg = torch.meshgrid(Q2, xs, indexing="ij")
    Qg, Xg = Qg.reshape(-1), Xg.reshape(-1)
    if points:
        Qg, Xg = Qg[:points], Xg[:points]
    area = DIS_SIGMA0_HALF_MB * MB_TO_GEV2

    def cfg(precision):
        return DISConfig(order=DISOrder.NLO, quarks=(Quark(QuarkType.LIGHT, 0.14),), transverse_area=area,
                         vegas_bins=DIS_BINS, precision=precision)

    opts = dict(vegas_samples=DIS_SAMPLES, vegas_iterations=DIS_ITERATIONS, vegas_min_iterations=DIS_ITERATIONS)
    # warm-up (compiles nothing; touches every kernel once)
    structure_functions(Qg[:2], Xg[:2], dipole, cfg("mixed"), sqrt_s=DIS_SQRT_S, seed=0,
                        vegas_samples=4096, vegas_iterations=2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    batch = structure_functions(Qg, Xg, dipole, cfg("mixed"), sqrt_s=DIS_SQRT_S, seed=0, **opts)
    stop.record()
    torch.cuda.synchronize()
    batch_s = start.elapsed_time(stop) / 1e3
    wall_s = time.perf_counter() - t0
    single_n = min(single, Qg.numel())
    t1 = time.perf_counter()
    singles = []
    for i in range(single_n):
        r = sigma_r(Qg[i].to(device), Xg[i].to(device), dipole, cfg("mixed"), sqrt_s=DIS_SQRT_S, seed=0, **opts)
        singles.append(float(r.value))
    torch.cuda.synchronize()
    single_s = (time.perf_counter() - t1) / max(single_n, 1)
    # FP64 build on the first points with the same Sobol points and seeds
    check_n = min(check, Qg.numel())
    fp64 = structure_functions(Qg[:check_n], Xg[:check_n], dipole, cfg("fp64"), sqrt_s=DIS_SQRT_S, seed=0, **opts)
    rel = (batch["sigma_r"][:check_n] - fp64["sigma_r"]).abs() / fp64["sigma_r"].abs()
    same = max(abs(singles[i] / float(batch["sigma_r"][i]) - 1) for i in range(single_n)) if single_n else None
    roofline = dis_nested_roofline(Qg, Xg, dipole, cfg("mixed"))
    line = {
        "metric": "DIS sigma_r points/s (NLO, batched)",
        "value": round(Qg.numel() / batch_s, 3),
        "unit": "points/s",
        "n_gpus": 1,
        "higher_is_better": True,
        "dtype": "f32+f64",
        "data": "synthetic: BK table evolved from the MV initial condition on the device",
        "config": {"workload": "NLO DIS sigma_r: 32 Q^2 in [1,50] x 16 x in [1e-5,1e-2], sqrt(s)=318, light quarks "
                               "m=0.14, sigma0/2=16 mb, Vegas 50 bins x 10 it x 2^18, seed 0",
                   "points": Qg.numel(), "integrals_per_point": 10},
        "batched_s": round(batch_s, 4),
        "batched_wall_s": round(wall_s, 4),
        "single_point_s": round(single_s, 4),
        "single_points_timed": single_n,
        "speedup_batched_vs_single": round(single_s / (batch_s / Qg.numel()), 3),
        "mixed_vs_fp64_max_rel": float(rel.max()) if check_n else None,
        "single_vs_batched_max_rel": same,
        "sigma_r_sample": [float(v) for v in batch["sigma_r"][:4]],
        "sigma_r_error_sample": [float(v) for v in batch["sigma_r_error"][:4]],
        "roofline": roofline,
    }
    return line


# Op census of one outer sample of the nested qqbar-g terms, from oracle/census_dis.py (an
# op-counting run of the DIS oracle's FP64 restatement; the mean of both polarisations):
# arithmetic = add, sub, mul, div; special = exp, log, sqrt, power, trigonometric, Bessel K0/K1.
DIS_CENSUS = {"I2N": {"arithmetic": 9866, "special": 3106}, "I3N": {"arithmetic": 9845, "special": 3091}}


def dis_nested_roofline(Qg, Xg, dipole, config) -> dict:
    """The nested I2 and I3 Vegas rounds of the DIS workload (all 512 points, both
    polarisations: 1,024 integrals, one round of 2^18 samples each), timed alone with CUDA
    events on their stream, against the census of the oracle restatement."""
    import torch

    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.dis import Polarization
    from nlo_bk_optimized_b200.dis.observables import kinematics
    from nlo_bk_optimized_b200.numerics.integration import VegasOptions, vegas_terms

    device = torch.device("cuda", 0)
    kins = [kinematics(float(q), float(x), pol, config, config.quarks[0])
            for q, x in zip(Qg.tolist(), Xg.tolist()) for pol in (Polarization.T, Polarization.L)]
    opts = VegasOptions(samples_per_iteration=DIS_SAMPLES, max_iterations=1, min_iterations=1, bins=DIS_BINS,
                        epsrel=1e-12)
    native = dipole.native()
    stream = torch.cuda.current_stream(device)
    out = {}
    flops = specials = seconds = 0.0
    for term in ("I2N", "I3N"):
        code = _native.DIS_TERMS[term]
        vegas_terms(code, kins[:2], native, opts, [0, 1], precision=_native.PRECISION_MIXED, device=device)  # warm
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(stream)
        vegas_terms(code, kins, native, opts, list(range(len(kins))), precision=_native.PRECISION_MIXED,
                    device=device)
        stop.record(stream)
        torch.cuda.synchronize()
        t = start.elapsed_time(stop) / 1e3
        n = len(kins) * DIS_SAMPLES
        out[term] = {"round_ms": round(t * 1e3, 3), "outer_samples": n}
        flops += n * DIS_CENSUS[term]["arithmetic"]
        specials += n * DIS_CENSUS[term]["special"]
        seconds += t
    sm_mhz = 1965.0
    peak = SM_COUNT * FP32_LANES_PER_SM * 2 * sm_mhz * 1e6 / 1e12
    mufu_peak = SM_COUNT * MUFU_PER_SM_PER_CLOCK * sm_mhz * 1e6
    achieved = flops / seconds / 1e12
    return {
        "bound": "fp32",
        "achieved": round(achieved, 3),
        "peak": round(peak, 2),
        "unit": "TFLOP/s",
        "frac": round(achieved / peak, 4),
        "traffic": None,
        "traffic_source": "not captured at the workload size; the kernel-case capture (one job, 2^16 samples) read "
                          "72-79 KB per launch: job arguments, grid and dipole table only",
        "kernel": "vegas_iteration_kernel<float, I2 nested / I3 nested> (csrc/dis.cu)",
        "peak_source": "nominal FP32 (148 SM x 128 lanes x 2 x 1965 MHz); MEASURED_PEAKS.json has only HBM and bf16",
        "census": {"source": "oracle/census_dis.py: op-counting run of the DIS oracle's FP64 nested integrands",
                   **DIS_CENSUS},
        "transcendental": {"achieved_per_s": round(specials / seconds, 1), "peak_per_s": mufu_peak,
                           "frac": round(specials / seconds / mufu_peak, 4),
                           "peak_source": "nominal 16 MUFU operations per SM per clock at 1965 MHz"},
        "rounds": out,
    }


# The reference's published C++ timings (20 CPU workers) of its six-term fixed-Sobol
# qqbar-g benchmark, benchmarks/dis_fixed_sobol_all_qg.py:69-76, in seconds.
FIXED_CPP_SECONDS = {"L_I1": 0.248004322, "L_I2": 0.315235827, "L_I3": 0.427307533,
                     "T_I1": 0.341898261, "T_I2": 0.932526175, "T_I3": 1.359838948}


def measure_fixed(reps: int = 20) -> dict:
    """The reference's fixed-Sobol qqbar-g benchmark setting (GBW Qs0^2 = 1, lambda = 0.3,
    gamma = 1, x0 = 1; charm m = 1.4; Q^2 = 9, x_Bj = 1e-3; maxr = 5, nf = 1; seed 3100):
    I1, I2 and I3 of both polarisations, one device call per polarisation (grid training on
    3 x 65,536 points, then 7 replicates of 32,768: 851,968 evaluations of the combined
    integrand), mixed precision.  Device time by CUDA events over `reps` repetitions, and
    end to end with the replicate estimates read back to the host."""
    import numpy as np
    import torch

    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.dipole import GBW
    from nlo_bk_optimized_b200.dis import DISConfig, Polarization, Quark, QuarkType
    from nlo_bk_optimized_b200.dis.fixed_sobol import fixed_sobol_device

    device = torch.device("cuda", torch.cuda.current_device())
    config = DISConfig(quarks=(Quark(QuarkType.C, 1.4),), maxr=5.0, nf_alphas=1, epsrel=0.001)
    dipole = GBW(Qs0sqr=1.0, lambda_=0.3, gamma=1.0, x0=1.0)
    pols = (("L", Polarization.L), ("T", Polarization.T))

    def run():
        return [fixed_sobol_device(9.0, 1e-3, pol, config.quarks[0], dipole, config, seed=3100, device=device,
                                   precision=_native.PRECISION_MIXED)[1] for _, pol in pols]

    for _ in range(3):
        run()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(reps):
        run()
    end.record(stream)
    torch.cuda.synchronize()
    device_s = start.elapsed_time(end) / 1000.0 / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        estimates = [e.cpu().numpy() for e in run()]
    e2e_s = (time.perf_counter() - t0) / reps
    terms = {}
    for (tag, _), est in zip(pols, estimates):
        for k in range(3):
            column = est[:, k]
            terms[f"{tag}_I{k + 1}"] = [float(column.mean()), float(column.std(ddof=1) / np.sqrt(column.size))]
    cpp = sum(FIXED_CPP_SECONDS.values())
    return {
        "metric": "six-term fixed-Sobol DIS qqbar-g evaluation (both polarisations, I1+I2+I3)",
        "value": round(device_s, 6),
        "unit": "s",
        "higher_is_better": False,
        "vs_baseline": round(device_s / cpp, 7),
        "baseline": {"value": round(cpp, 6), "unit": "s",
                     "source": "reference C++ on 20 CPU workers, benchmarks/dis_fixed_sobol_all_qg.py:69-76; "
                               "the reference's own GPU path is quoted at 186-189x faster (RTX 3090)"},
        "speedup_vs_cpp": round(cpp / device_s, 1),
        "e2e": {"value": round(e2e_s, 6), "unit": "s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 2 * 7 * 3 * 8},
        "dtype": "f32+f64",
        "data": "synthetic: the reference benchmark's GBW charm setting",
        "config": {"workload": "GBW(1, 0.3, 1, 1), charm m=1.4, Q^2=9, x=1e-3, maxr=5, nf=1, seed 3100; "
                               "3 x 2^16 training + 7 x 2^15 replicate Sobol points per polarisation",
                   "reps": reps},
        "terms": terms,
    }


def run_fixed(args) -> None:
    print(json.dumps(measure_fixed()))


def run_dis(args) -> None:
    print(json.dumps(measure_dis(args.dis_points, args.dis_single, args.dis_check)))


# ---------------------------------------------------------------------------
# Batched and served workloads: parameter sets drawn from a seeded generator
# (Qs0^2 ~ U[0.05, 0.5], gamma ~ U[0.8, 1.3], e_c ~ logU[1, 100]), each evolved with the
# 200-point grid in [1e-6, 1e2] (RK4, h = 0.2, frozen-coupling cap 0.7) and uneven Monte
# Carlo budgets 2^U{16..20} Sobol points per r per stage.

def _sets(n: int, seed: int = 0):
    import torch

    g = torch.Generator().manual_seed(seed)
    u = torch.rand((n, 4), generator=g, dtype=torch.float64)
    qs = 0.05 + 0.45 * u[:, 0]
    gamma = 0.8 + 0.5 * u[:, 1]
    ec = torch.exp(u[:, 2] * math.log(100.0))
    budgets = (2 ** (16 + torch.floor(u[:, 3] * 5))).to(torch.int64)
    return [(float(qs[i]), float(gamma[i]), float(ec[i]), int(budgets[i])) for i in range(n)]


def _small_bk_config(samples: int = 1 << 16):
    from nlo_bk_optimized_b200 import BKConfig
    from nlo_bk_optimized_b200.bk.config import IntegrationMethod

    return BKConfig(RPOINTS=199, MINR=1e-6, MAXR=1e2, MCINTPOINTS=samples, DE_SOLVER_STEP=0.2, STEPPER="rk4",
                    PRECISION="mixed", ALPHA_S_CAP=0.7, INTMETHOD_NLO=IntegrationMethod.SOBOL)


def _set_points(k: int, count: int = 8) -> list[tuple[float, float]]:
    """The DIS points of parameter set k: Q^2 log-uniform in [1, 50] GeV^2 and x_Bj log-uniform
    in [1e-2, 5e-2] (seeded by k), inside the rapidity range of a table evolved to Y = 4 from
    x0 = 0.01: ln(Q^2 / (x Q0^2)) <= 8.52 < 4 + ln(1/x0)."""
    import torch

    g = torch.Generator().manual_seed(1000 + k)
    u = torch.rand((count, 2), generator=g, dtype=torch.float64)
    Q2 = torch.exp(u[:, 0] * math.log(50.0))
    xs = 1e-2 * torch.exp(u[:, 1] * math.log(5.0))
    return [(float(q), float(x)) for q, x in zip(Q2, xs)]


BATCH_MAXY = 4.0  # the evolution of the batched parameter sets: RK4, h = 0.2, to Y = 4


def measure_batch(n_sets: int) -> dict:
    """The batched solve: n_sets MV parameter sets (Qs0^2 ~ U[0.05, 0.5], gamma ~ U[0.8, 1.3],
    e_c ~ logU[1, 100], budgets 2^U{16..20} Sobol points per r per stage) evolved on 200 r in
    [1e-6, 1e2] (RK4 h = 0.2 to Y = 4, alpha_s capped at 0.7), then each set's 8 (Q^2, x_Bj)
    points (NLO F_T, F_L, F_2, sigma_r at sqrt(s) = 318 GeV, light quarks, Vegas of 4
    iterations x budget/16 samples) -- all evolutions in one multi-set evolution (one launch per
    kernel and stage for every set) and all points of all sets in one merged DIS run -- against
    the plain single-solve path
    (solve_bk of one set, then sigma_r of one point at a time), timed on one set of each
    budget class and summed over the classes' set counts."""
    import torch

    from nlo_bk_optimized_b200 import MV, solve_bk
    from nlo_bk_optimized_b200.bk.batch import evolve_batch, tune_waves
    from nlo_bk_optimized_b200.bk.evolution import _r_grid, _steps_to
    from nlo_bk_optimized_b200.dipole import BKDipole, DipoleTable
    from nlo_bk_optimized_b200.dis import DISConfig, DISOrder, Quark, QuarkType, sigma_r, structure_functions
    from nlo_bk_optimized_b200.dis import structure_functions_many
    from nlo_bk_optimized_b200.serving import dis_options_for

    device = torch.device("cuda", 0)
    sets = _sets(n_sets)
    config = _small_bk_config()
    dis = DISConfig(order=DISOrder.NLO, quarks=(Quark(QuarkType.LIGHT, 0.14),))
    r_host = _r_grid(config, device="cpu", dtype=torch.float64)
    N0 = torch.stack([MV(qs0sqr=q, gamma=g, ec=e).dipole_amplitude(r_host).to(torch.float64)
                      for q, g, e, _ in sets]).to(device)
    r = r_host.to(device)
    budgets = [b for *_, b in sets]
    ys = _steps_to(0.0, BATCH_MAXY, 0.2)
    y = torch.tensor([0.0, *ys], dtype=torch.float64, device=device)
    points = [_set_points(k) for k in range(n_sets)]

    marks = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

    def batched():
        marks[0].record()
        tables = evolve_batch(N0, r, len(ys), config, budgets, waves=waves)
        marks[1].record()
        dipoles = [BKDipole(DipoleTable(r=r, y=y, N=tables[k], x0=0.01)) for k in range(n_sets)]
        Q2 = [q for pts in points for q, _ in pts]
        xs = [x for pts in points for _, x in pts]
        dips = [dipoles[k] for k, pts in enumerate(points) for _ in pts]
        seeds = [k for k, pts in enumerate(points) for _ in pts]
        opts = [dis_options_for(budgets[k]) for k, pts in enumerate(points) for _ in pts]
        out = structure_functions_many(Q2, xs, dips, dis, sqrt_s=DIS_SQRT_S, seeds=seeds, options=opts)
        marks[2].record()
        return out["sigma_r"].cpu()

    waves = tune_waves(N0, r, config, budgets)
    # warm-up of every kernel on the path: a short evolution of two sets and two of their points
    warm = evolve_batch(N0[:2], r, len(ys), config, [1 << 10] * 2, waves=waves)
    warm_dipoles = [BKDipole(DipoleTable(r=r, y=y, N=warm[k], x0=0.01)) for k in range(2)]
    structure_functions_many([points[0][0][0], points[1][0][0]], [points[0][0][1], points[1][0][1]], warm_dipoles,
                             dis, sqrt_s=DIS_SQRT_S, seeds=[0, 1], options=[dis_options_for(1 << 16)] * 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sig_batched = batched()
    torch.cuda.synchronize()
    batched_s = time.perf_counter() - t0
    split = (marks[0].elapsed_time(marks[1]) / 1e3, marks[1].elapsed_time(marks[2]) / 1e3)

    # the evolution alone (the same multi-set call) and its K2+Kf evaluations: budget x active
    # parents of each step's row, four right-hand sides a step
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tables = evolve_batch(N0, r, len(ys), config, budgets, waves=waves)
    torch.cuda.synchronize()
    evolve_s = time.perf_counter() - t0
    active = (tables[:, :-1, 1:] <= 0.99999).sum(dim=2).to(torch.float64)  # [sets, steps]
    k2kf_evals = float((active.sum(dim=1) * torch.tensor(budgets, dtype=torch.float64, device=device)).sum()) * 4

    # the plain path on one set of each budget class
    classes: dict[int, list[int]] = {}
    for k, b in enumerate(budgets):
        classes.setdefault(b, []).append(k)
    per_class_point, per_class_set = {}, {}
    ic_of = lambda k: MV(qs0sqr=sets[k][0], gamma=sets[k][1], ec=sets[k][2])  # noqa: E731
    single_vs_batched = 0.0
    # the plain path's own warm-up (its first solve_bk and sigma_r load what they need)
    warm_table = BKDipole(solve_bk(ic_of(0), BATCH_MAXY, _small_bk_config(1 << 10), device=device,
                                   dtype=torch.float64, seed=0))
    sigma_r(torch.tensor(points[0][0][0], dtype=torch.float64, device=device),
            torch.tensor(points[0][0][1], dtype=torch.float64, device=device), warm_table, dis, sqrt_s=DIS_SQRT_S,
            seed=0, **dis_options_for(1 << 16))
    structure_functions(torch.tensor([points[0][0][0]], dtype=torch.float64),
                        torch.tensor([points[0][0][1]], dtype=torch.float64), warm_table, dis, sqrt_s=DIS_SQRT_S,
                        seed=0, **dis_options_for(1 << 16))["sigma_r"].cpu()
    for b, members in sorted(classes.items()):
        k = members[0]
        cfg = _small_bk_config(b)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        table = solve_bk(ic_of(k), BATCH_MAXY, cfg, device=device, dtype=torch.float64, seed=0)
        dipole = BKDipole(table)
        vals = []
        for j, (q2, x) in enumerate(points[k]):
            res = sigma_r(torch.tensor(q2, dtype=torch.float64, device=device),
                          torch.tensor(x, dtype=torch.float64, device=device), dipole, dis, sqrt_s=DIS_SQRT_S,
                          seed=k, **dis_options_for(b))
            vals.append(float(res.value))
        torch.cuda.synchronize()
        per_class_point[b] = time.perf_counter() - t0
        t0 = time.perf_counter()
        sf = structure_functions(torch.tensor([q for q, _ in points[k]], dtype=torch.float64),
                                 torch.tensor([x for _, x in points[k]], dtype=torch.float64),
                                 BKDipole(solve_bk(ic_of(k), BATCH_MAXY, cfg, device=device, dtype=torch.float64,
                                                   seed=0)), dis, sqrt_s=DIS_SQRT_S, seed=k, **dis_options_for(b))
        sf["sigma_r"].cpu()
        per_class_set[b] = time.perf_counter() - t0
        base = sum(len(p) for p in points[:k])
        for j, v in enumerate(vals):
            single_vs_batched = max(single_vs_batched, abs(v / float(sig_batched[base + j]) - 1))
    plain_points = sum(per_class_point[b] * len(m) for b, m in classes.items())
    plain_sets = sum(per_class_set[b] * len(m) for b, m in classes.items())
    n_points = sum(len(p) for p in points)
    return {
        "metric": "batched NLO BK + DIS: parameter sets evolved and evaluated per second",
        "value": round(n_sets / batched_s, 3),
        "unit": "parameter sets/s",
        "n_gpus": 1,
        "higher_is_better": True,
        "dtype": "f32+f64",
        "data": "synthetic: MV parameter sets from torch.Generator().manual_seed(0), seeded DIS points",
        "config": {"workload": f"{n_sets} MV sets, 200 r in [1e-6,1e2], RK4 h=0.2 to Y={BATCH_MAXY}, alpha_s cap 0.7, "
                               "budgets 2^U{16..20} per r per stage; 8 (Q^2,x) points per set, NLO sigma_r, "
                               "Vegas 4 it x budget/16", "sets": n_sets, "points": n_points, "waves": waves},
        "batched_s": round(batched_s, 3),
        "batched_split_s": {"evolution": round(split[0], 3), "dis": round(split[1], 3)},
        "evolution_s": round(evolve_s, 3),
        "evolution_k2kf_evals": k2kf_evals,
        "evolution_k2kf_evals_per_s": round(k2kf_evals / evolve_s, 1),
        "dis_points_per_s": round(n_points / batched_s, 2),
        "plain_single_point_s": round(plain_points, 2),
        "plain_single_point_per_set_s": {str(b): round(t, 4) for b, t in sorted(per_class_point.items())},
        "speedup_vs_plain_single_point": round(plain_points / batched_s, 3),
        "plain_per_set_s": round(plain_sets, 2),
        "speedup_vs_plain_per_set": round(plain_sets / batched_s, 3),
        "plain_timing": "one set of each budget class timed, times its class's set count",
        "single_vs_batched_max_rel": single_vs_batched,
    }


def run_batch(args) -> None:
    print(json.dumps(measure_batch(args.batch_sets)))


def _requests_for(seconds: float, rate: float, seed: int = 0):
    import random

    from nlo_bk_optimized_b200.serving import Request

    rng = random.Random(seed)
    sets = _sets(4096, seed=1)
    Q2s = [1.0 * (50.0 ** (k / 31)) for k in range(32)]
    xs = [1e-3 * (10.0 ** (k / 15)) for k in range(16)]
    grid = [(q, x) for q in Q2s for x in xs]
    t, requests = 0.0, []
    while t < seconds:
        t += rng.expovariate(rate)
        q, g, e, _ = sets[len(requests) % len(sets)]
        budget = int(round(2 ** rng.uniform(16, 20)))  # log-uniform in [2^16, 2^20]
        pts = tuple(rng.sample(grid, rng.randint(1, 64)))
        requests.append((t, Request(q, g, e, pts, budget, seed=len(requests))))
    return requests


def measure_serve(seconds: float, rate: float, slots: int, waves: int, sample: int = 24) -> dict:
    """Poisson arrivals at `rate`/s for `seconds`: each request is one parameter set (drawn as
    in the batched workload), 1-64 points of the 32 x 16 DIS grid restricted to x >= 1e-3 and
    an MC budget log-uniform in [2^16, 2^20].  p50/p99 latency and points/s of the server
    (continuous batching) against the same requests run one at a time through the plain
    single-solve path (a sample of them)."""
    import torch

    from nlo_bk_optimized_b200.dis import DISConfig, DISOrder, Quark, QuarkType
    from nlo_bk_optimized_b200.serving import Server, run_alone

    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    requests = _requests_for(seconds, rate)
    bk = _small_bk_config()
    dis = DISConfig(order=DISOrder.NLO, quarks=(Quark(QuarkType.LIGHT, 0.14),))
    run_alone(requests[0][1], bk, dis)  # warm-up
    server = Server(bk, dis, slots=slots, waves=waves)
    t0 = time.perf_counter()
    futures = []
    for at, req in requests:
        delay = at - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        futures.append(server.submit(req))
    for f in futures:
        f.result()
    server.close()
    served = server.stats.summary()
    pick = requests[:: max(1, len(requests) // sample)][:sample]
    t1 = time.perf_counter()
    for _, req in pick:
        run_alone(req, bk, dis)
    alone = (time.perf_counter() - t1) / len(pick)
    alone_pts = sum(len(r.points) for _, r in pick) / len(pick)
    sequential_pps = alone_pts / alone
    # requests of 1-64 points: the sample's points per request differ from the population's, so
    # the request rate is compared too (a request's cost is mostly its evolution)
    return {
        "metric": "served NLO BK + DIS requests: p50/p99 latency and points/s",
        "value": round(served["points_per_s"], 3),
        "unit": "points/s",
        "n_gpus": 1,
        "higher_is_better": True,
        "dtype": "f32+f64",
        "data": "synthetic Poisson arrivals, seeded",
        "config": {"workload": f"Poisson {rate}/s for {seconds} s, 1-64 points per request, budgets logU[2^16, 2^20]",
                   "slots": slots, "waves": waves, "requests": len(requests)},
        "p50_s": served["p50_s"],
        "p99_s": served["p99_s"],
        "requests_per_s": served["requests_per_s"],
        "engine_steps": len(server.step_sets),
        "mean_evolutions_per_engine_step": round(sum(server.step_sets) / max(1, len(server.step_sets)), 2),
        "dis_batches": len(server.batches),
        "mean_requests_per_dis_batch": round(sum(server.batches) / max(1, len(server.batches)), 2),
        "sequential_points_per_s": round(sequential_pps, 3),
        "sequential_request_s_mean": round(alone, 4),
        "sequential_sample": len(pick),
        "speedup_vs_sequential": round(served["points_per_s"] / sequential_pps, 3),
        "speedup_vs_sequential_requests": round(served["requests_per_s"] * alone, 3),
        "sequential_points_per_request": round(alone_pts, 2),
        "served_points_per_request": round(served["points"] / max(1, served["requests"]), 2),
    }


def run_serve(args) -> None:
    print(json.dumps(measure_serve(args.serve_seconds, args.serve_rate, args.serve_slots, args.serve_waves)))


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--e2e-steps", type=int, default=5, help="whole evolutions timed through solve_bk")
    parser.add_argument("--kernel-case", action="store_true",
                        help="run only the small K2+Kf/K1 case used for ncu captures")
    parser.add_argument("--workload", choices=["bk", "dis", "fixed", "batch", "serve"], default="bk",
                        help="bk: the NLO BK evolution (default); dis: NLO DIS sigma_r throughput; fixed: the "
                             "reference's fixed-Sobol qqbar-g benchmark; batch: many parameter sets at once; "
                             "serve: the request loop under Poisson arrivals")
    parser.add_argument("--batch-sets", type=int, default=256)
    parser.add_argument("--batch-maxy", type=float, default=8.0)
    parser.add_argument("--serve-rate", type=float, default=200.0)
    parser.add_argument("--serve-seconds", type=float, default=1.0)
    parser.add_argument("--serve-slots", type=int, default=64)
    parser.add_argument("--serve-waves", type=int, default=4)
    parser.add_argument("--no-batch", action="store_true", help="skip the batched and served objects of the line")
    parser.add_argument("--line-batch-sets", type=int, default=32, help="parameter sets of the line's batch object")
    parser.add_argument("--line-serve-seconds", type=float, default=0.5, help="arrival window of the line's serve object")
    parser.add_argument("--no-dis", action="store_true", help="skip the DIS sigma_r measurement")
    parser.add_argument("--dis-points", type=int, default=0, help="DIS: first N of the 512 points (0 = all)")
    parser.add_argument("--dis-single", type=int, default=4, help="DIS: points timed through single sigma_r calls")
    parser.add_argument("--dis-check", type=int, default=4, help="DIS: points recomputed in FP64")
    args = parser.parse_args()
    if args.workload == "batch":
        run_batch(args)
        return
    if args.workload == "serve":
        run_serve(args)
        return
    if args.workload == "fixed":
        run_fixed(args)
        return
    if args.workload == "dis":
        if args.kernel_case:
            run_dis_kernel_case()
        else:
            run_dis(args)
        return
    if args.kernel_case:
        run_kernel_case()
        return
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
