"""Many BK evolutions at once: independent parameter sets with uneven Monte Carlo budgets.

All sets of a call advance together through one ``nlo_bk_evolve_sets`` call (the whole
rapidity loop in C, no host synchronisation): every stage is one launch per kernel for all
sets, and the K2+Kf launch gives its lanes (set, parent) pairs -- a CTA stages one tile of
sample records per set it holds, and sets of equal budget share CTAs, so small budgets no
longer pay a whole under-filled launch each.  Each set has its own Sobol seed (a set of budget
S uses the first S points of its sequence).  The K2+Kf launch takes about ``waves`` x 2 CTAs
per SM, spread over the sets' groups -- which fixes the sample chunk each CTA sweeps -- and
``tune_waves`` picks ``waves`` by timing one rapidity step of a sample of the sets at each
candidate.  A set's rows equal ``solve_bk``'s for the same initial row, budget and seed up to
the order in which the FP64 partial sums of the CTAs are added.
"""

from __future__ import annotations

import ctypes
import time
from collections.abc import Sequence

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.bk.config import BKConfig, require_fixed_step, require_sobol
from nlo_bk_optimized_b200.dipole.table import DipoleTable

WAVE_CHOICES = (1, 2, 4, 8, 16)
DEFAULT_WAVES = 4
MAX_SETS = 256  # sets per nlo_bk_evolve_sets call


def evolve_batch(N0: torch.Tensor, r: torch.Tensor, steps: int, config: BKConfig, samples: Sequence[int], *,
                 seed: int = 0, seeds: Sequence[int] | None = None, waves: int = DEFAULT_WAVES,
                 precision: int | None = None) -> torch.Tensor:
    """Rows [B, steps+1, R] (float64, on the device of r) for initial rows N0 [B, R]; set b
    takes Sobol seed ``seeds[b]`` (default: ``seed`` for every set)."""
    from nlo_bk_optimized_b200.bk.evolution import nlo_box, params_of, precision_of

    require_sobol(config, "the batched evolution")
    require_fixed_step(config, "the batched evolution")
    if config.KINEMATICAL_CONSTRAINT:
        raise NotImplementedError("the kinematical constraint is not available for the batched evolution")
    device = r.device
    B, points = N0.shape
    if len(samples) != B:
        raise ValueError("one Monte Carlo budget per parameter set is required")
    if any(int(s) < 0 or int(s) > 1 << 30 for s in samples):
        raise ValueError("budgets must lie in [0, 2^30]")
    lib = _native.load()
    prec = precision if precision is not None else precision_of(config, torch.float32)
    params = params_of(config, prec)
    lower, width = nlo_box(float(r[0]), float(r[-1]))
    box = _native.box(lower, width)
    seeds = [int(seed)] * B if seeds is None else [int(v) for v in seeds]
    if len(seeds) != B:
        raise ValueError("one seed per parameter set is required")
    dirs_of = {v: _native.sobol_dirs(4, v) for v in set(seeds)}
    stepper = _native.STEPPERS[config.stepper]
    tables = torch.empty((B, steps + 1, points), dtype=torch.float64, device=device)
    tables[:, 0] = N0
    status = torch.zeros(B, dtype=torch.int32, device=device)  # one word per set
    r = r.to(torch.float64).contiguous()
    stream = torch.cuda.current_stream(device).cuda_stream
    with torch.cuda.device(device):
        for start in range(0, B, MAX_SETS):
            n = min(MAX_SETS, B - start)
            workspace = torch.empty(int(lib.nlo_bk_sets_workspace_bytes(points, n, waves)), dtype=torch.uint8,
                                    device=device)
            ptrs = (ctypes.c_void_p * n)(*[tables[start + k].data_ptr() for k in range(n)])
            budgets = (ctypes.c_int64 * n)(*[int(samples[start + k]) for k in range(n)])
            dirs = (_native.SobolDirs * n)(*[dirs_of[seeds[start + k]] for k in range(n)])
            _native.check(lib.nlo_bk_evolve_sets(params, r.data_ptr(), points, n, ptrs, steps,
                                                 float(config.DE_SOLVER_STEP), stepper, dirs, budgets, box, waves,
                                                 status[start:].data_ptr(), workspace.data_ptr(), workspace.numel(),
                                                 stream))
    if bool(status.any()):
        raise FloatingPointError("non-finite BK amplitude during a batched evolution")
    return tables


def tune_waves(N0: torch.Tensor, r: torch.Tensor, config: BKConfig, samples: Sequence[int], *,
               sample_sets: int = 32, choices: Sequence[int] = WAVE_CHOICES, precision: int | None = None) -> int:
    """Pick the K2+Kf CTA count (``waves``) that evolves a sample of the sets one rapidity step
    fastest.  Each candidate runs once untimed first, so that its workspace (whose size grows
    with ``waves``) is allocated outside the timed call."""
    pick = list(range(0, N0.shape[0], max(1, N0.shape[0] // sample_sets)))[:sample_sets]
    N = N0[pick]
    S = [samples[i] for i in pick]
    best, best_t = choices[0], float("inf")
    for c in choices:
        evolve_batch(N, r, 1, config, S, waves=c, precision=precision)
        torch.cuda.synchronize(r.device)
        t0 = time.perf_counter()
        evolve_batch(N, r, 1, config, S, waves=c, precision=precision)
        torch.cuda.synchronize(r.device)
        t = time.perf_counter() - t0
        if t < best_t:
            best, best_t = c, t
    return best


def solve_bk_batch(initial_conditions: Sequence, maxy: float, config: BKConfig = BKConfig(), *,
                   samples: Sequence[int] | None = None, device: torch.device | str = "cuda",
                   dtype: torch.dtype = torch.float32, seed: int = 0, waves: int | None = None) -> list[DipoleTable]:
    """``solve_bk`` for many initial conditions; ``samples[i]`` overrides MCINTPOINTS of set i.
    ``waves=None`` lets ``tune_waves`` choose the K2+Kf CTA count."""
    from nlo_bk_optimized_b200.bk.evolution import _cuda_device, _r_grid, _steps_to, initial_row, precision_of

    device = _cuda_device(device)
    if not initial_conditions:
        return []
    budgets = list(samples) if samples is not None else [int(config.MCINTPOINTS)] * len(initial_conditions)
    r_host = _r_grid(config, device="cpu", dtype=torch.float64)
    N0 = torch.stack([initial_row(ic, r_host, device) for ic in initial_conditions])
    r = r_host.to(device)
    ys = _steps_to(0.0, maxy, config.DE_SOLVER_STEP)
    precision = precision_of(config, dtype)
    if waves is None:
        waves = tune_waves(N0, r, config, budgets, precision=precision)
    tables = evolve_batch(N0, r, len(ys), config, budgets, seed=seed, waves=waves, precision=precision)
    y = torch.tensor([0.0, *ys], dtype=dtype, device=device)
    return [DipoleTable(r=r.to(dtype), y=y, N=tables[b].to(dtype), x0=ic.x0)
            for b, ic in enumerate(initial_conditions)]


__all__ = ["evolve_batch", "solve_bk_batch", "tune_waves"]
