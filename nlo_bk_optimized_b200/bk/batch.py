"""Many BK evolutions at once: independent parameter sets with uneven Monte Carlo budgets.

Each set is one ``nlo_bk_evolve`` call (the whole rapidity loop in C, no host
synchronisation) on one of several CUDA streams, issued by one host thread per stream
(the ctypes calls release the interpreter lock), each stream with its own workspace and
status word.  Kernels of different sets overlap on the GPU, so sets with small budgets --
whose launches alone would leave most SMs idle -- fill each other's gaps.  The number of
streams is chosen by ``tune_streams``, which times one rapidity step of a sample of the
sets at each candidate concurrency.
"""

from __future__ import annotations

import time
from collections.abc import Sequence
from concurrent.futures import ThreadPoolExecutor

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.bk.config import BKConfig, require_sobol
from nlo_bk_optimized_b200.dipole.table import DipoleTable

STREAM_CHOICES = (1, 2, 4, 8, 16)


class _Lane:
    """A stream with its own workspace."""

    def __init__(self, device: torch.device, points: int):
        lib = _native.load()
        self.stream = torch.cuda.Stream(device=device)
        self.workspace = torch.empty(int(lib.nlo_bk_rhs_workspace_bytes(points)), dtype=torch.uint8, device=device)


def _evolve_set(lib, lane: _Lane, params, r: torch.Tensor, table: torch.Tensor, status: torch.Tensor, steps: int,
                step: float, stepper: int, dirs, samples: int, box) -> None:
    _native.check(lib.nlo_bk_evolve(params, r.data_ptr(), r.numel(), steps, step, stepper, dirs, int(samples), box,
                                    table.data_ptr(), status.data_ptr(), lane.workspace.data_ptr(),
                                    lane.workspace.numel(), lane.stream.cuda_stream))


def evolve_batch(N0: torch.Tensor, r: torch.Tensor, steps: int, config: BKConfig, samples: Sequence[int], *,
                 seed: int = 0, streams: int = 8, precision: int | None = None) -> torch.Tensor:
    """Rows [B, steps+1, R] (float64, on the device of r) for initial rows N0 [B, R]."""
    from nlo_bk_optimized_b200.bk.evolution import nlo_box, params_of, precision_of

    require_sobol(config, "the batched evolution")
    device = r.device
    B, points = N0.shape
    if len(samples) != B:
        raise ValueError("one Monte Carlo budget per parameter set is required")
    lib = _native.load()
    prec = precision if precision is not None else precision_of(config, torch.float32)
    params = params_of(config, prec)
    lower, width = nlo_box(float(r[0]), float(r[-1]))
    box = _native.box(lower, width)
    dirs = _native.sobol_dirs(4, seed)
    stepper = _native.STEPPERS[config.stepper]
    tables = torch.empty((B, steps + 1, points), dtype=torch.float64, device=device)
    tables[:, 0] = N0
    status = torch.zeros(B, dtype=torch.int32, device=device)  # one word per set
    streams = max(1, min(streams, B))
    lanes = [_Lane(device, points) for _ in range(streams)]
    start = torch.cuda.current_stream(device)
    for lane in lanes:
        lane.stream.wait_stream(start)

    def issue(k: int) -> None:
        with torch.cuda.device(device):
            for b in range(k, B, streams):
                _evolve_set(lib, lanes[k], params, r, tables[b], status[b:b + 1], steps,
                            float(config.DE_SOLVER_STEP), stepper, dirs, samples[b], box)

    with ThreadPoolExecutor(max_workers=streams) as pool:
        list(pool.map(issue, range(streams)))
    for lane in lanes:
        start.wait_stream(lane.stream)
    if bool(status.any()):
        raise FloatingPointError("non-finite BK amplitude during a batched evolution")
    return tables


def tune_streams(N0: torch.Tensor, r: torch.Tensor, config: BKConfig, samples: Sequence[int], *,
                 sample_sets: int = 32, choices: Sequence[int] = STREAM_CHOICES, precision: int | None = None) -> int:
    """Pick the stream count that evolves a sample of the sets (one rapidity step) fastest."""
    pick = list(range(0, N0.shape[0], max(1, N0.shape[0] // sample_sets)))[:sample_sets]
    N = N0[pick]
    S = [samples[i] for i in pick]
    best, best_t = choices[0], float("inf")
    evolve_batch(N[:1], r, 1, config, S[:1], streams=1, precision=precision)  # load kernels before timing
    for c in choices:
        torch.cuda.synchronize(r.device)
        t0 = time.perf_counter()
        evolve_batch(N, r, 1, config, S, streams=c, precision=precision)
        torch.cuda.synchronize(r.device)
        t = time.perf_counter() - t0
        if t < best_t:
            best, best_t = c, t
    return best


def solve_bk_batch(initial_conditions: Sequence, maxy: float, config: BKConfig = BKConfig(), *,
                   samples: Sequence[int] | None = None, device: torch.device | str = "cuda",
                   dtype: torch.dtype = torch.float32, seed: int = 0, streams: int | None = None) -> list[DipoleTable]:
    """``solve_bk`` for many initial conditions; ``samples[i]`` overrides MCINTPOINTS of set i.
    ``streams=None`` lets ``tune_streams`` choose the concurrency."""
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
    if streams is None:
        streams = tune_streams(N0, r, config, budgets, precision=precision)
    tables = evolve_batch(N0, r, len(ys), config, budgets, seed=seed, streams=streams, precision=precision)
    y = torch.tensor([0.0, *ys], dtype=dtype, device=device)
    return [DipoleTable(r=r.to(dtype), y=y, N=tables[b].to(dtype), x0=ic.x0)
            for b, ic in enumerate(initial_conditions)]


__all__ = ["evolve_batch", "solve_bk_batch", "tune_streams"]
