"""BK rapidity evolution on the B200 (mirrors torch_nlo_clean/src/nlo_torch/bk/evolution.py).

``solve_bk`` / ``compute_dndy`` keep the reference signatures.  The whole
evolution runs on one CUDA stream through ``nlo_bk_evolve`` (K2+Kf by scrambled Sobol
QMC) or ``nlo_bk_evolve_vegas`` (K2+Kf by Vegas per parent, the reference's default) of
libnlo_b200.so: per stage a FP64 spline refit, K1 (fixed 8 x 24 rule), K2+Kf and the FP64
RK combination -- no host synchronisation between stages.  The host reads back once, at
the end, to check the non-finite flag (bk/evolution.py:152-153 raises
FloatingPointError).  The Vegas grids of one evolution (one per parent) live in a device
buffer that the whole evolution shares, like the reference's per-parent vegas_states of
one _bk_steps run (bk/evolution.py:85-100).
"""

from __future__ import annotations

import ctypes
import math
from collections.abc import Iterator
from dataclasses import dataclass

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.bk.config import (
    ORDER_CODES,
    RC_LO_CODES,
    RC_NLO_CODES,
    RESUM_RC_CODES,
    BKConfig,
    IntegrationMethod,
    device_supported,
    fixed_coupling,
)
from nlo_bk_optimized_b200.bk.initial_conditions import MV, ICDataFile
from nlo_bk_optimized_b200.dipole.table import DipoleTable


@dataclass(frozen=True, slots=True)
class DNDYResult:
    r: torch.Tensor
    K1: torch.Tensor
    K2_Kf: torch.Tensor
    N: torch.Tensor


def _r_grid(config: BKConfig, *, device: torch.device | str, dtype: torch.dtype) -> torch.Tensor:
    """r_i = MINR (MAXR/MINR)^(i/RPOINTS), i = 0..RPOINTS (bk/evolution.py:584-592)."""

    rind = torch.arange(config.RPOINTS + 1, dtype=dtype, device=device)
    step = (config.MAXR / config.MINR) ** (1 / config.RPOINTS)
    return config.MINR * torch.pow(rind.new_tensor(step), rind)


def nlo_box(r_first: float, r_last: float) -> tuple[list[float], list[float]]:
    """[log(r0/2), log(2 r_max)]^2 x [0, 2 pi]^2 (bk/derivatives.py:424-431) as (lower, width)."""

    lo = math.log(0.5 * r_first)
    hi = math.log(2 * r_last)
    return [lo, lo, 0.0, 0.0], [hi - lo, hi - lo, 2 * math.pi, 2 * math.pi]


def precision_of(config: BKConfig, dtype: torch.dtype) -> int:
    choice = config.PRECISION or ("mixed" if dtype == torch.float32 else "fp64")
    return _native.PRECISION_FP64 if choice == "fp64" else _native.PRECISION_MIXED


def params_of(config: BKConfig, precision: int) -> _native.BKParams:
    reason = device_supported(config)
    if reason is not None:
        raise NotImplementedError(reason)
    p = _native.BKParams()
    p.nc = float(config.NC)
    p.nf = float(config.NF)
    p.lambda_qcd = float(config.LambdaQCD)
    p.c2 = float(config.C2)
    p.minr = float(config.MINR)
    p.ksub = float(config.KSUB)
    p.fixed_alpha_s = float(config.FIXED_AS)
    p.alpha_cap = float(config.ALPHA_S_CAP)
    p.symmetrize = int(bool(config.SYMMETRIZE_Z_Z2_INTEGRATION))
    p.fixed_coupling = int(fixed_coupling(config))
    p.force_positive = int(bool(config.FORCE_POSITIVE_N))
    p.precision = int(precision)
    p.order = ORDER_CODES[config.Order]
    p.rc_lo = RC_LO_CODES[config.RC_LO]
    p.resum_rc = RESUM_RC_CODES[config.RESUM_RC]
    p.rc_nlo = RC_NLO_CODES[config.RC_NLO]
    p.kinematical_constraint = int(bool(config.KINEMATICAL_CONSTRAINT))
    return p


VEGAS_BINS = 32


def vegas_options_of(config: BKConfig) -> _native.BKVegasOptions | None:
    """The Vegas settings of rapidity_derivative_nlo (bk/derivatives.py:389-421) for
    IntegrationMethod.VEGAS: MCINTPOINTS per iteration, a warm-up of max(2, MCINTPOINTS/5),
    2..4 iterations, 32 bins, epsrel 0.2, and the grid reuse of BKConfig; None otherwise."""
    if config.INTMETHOD_NLO is not IntegrationMethod.VEGAS:
        return None
    o = _native.BKVegasOptions()
    o.samples_per_iteration = int(config.MCINTPOINTS)
    o.warmup_samples = max(2, int(config.MCINTPOINTS) // 5)
    o.max_iterations = 4
    o.min_iterations = 2
    o.bins = VEGAS_BINS
    o.reuse_grid = int(bool(config.VEGAS_REUSE_GRID))
    o.reuse_warmup_fraction = float(config.VEGAS_REUSE_WARMUP_FRACTION)
    o.epsrel = 0.2
    o.epsabs = 0.0
    return o


VEGAS_REPLICAS = 6  # bk/evolution.py:437: replicas 1..6 with seeds seed + 1000 k


def vegas_evolution_setup(config: BKConfig, seed: int | None):
    """Options and direction sets of an evolution with K2+Kf by Vegas: the replica refinement of
    bk/evolution.py:411-456 runs where the reference's evolution keeps per-parent grids
    (VEGAS_REUSE_GRID) and a seed is given -- 6 more integrals on fresh grids with the seeds
    seed + 1000 k for a parent whose K1 and K2, Kf cancel strongly or whose N exceeds 0.9.  The
    reference does this on its CUDA float32 path; both builds here do it, so that the all-FP64
    build checks the mixed one.  Returns (options, dirs array of 1 + replicas), or (None, dirs)
    for the QMC integrator."""
    base = 0 if seed is None else int(seed)
    opts = vegas_options_of(config)
    replicas = VEGAS_REPLICAS if (opts is not None and seed is not None and opts.reuse_grid) else 0
    if opts is not None:
        opts.replicas = replicas
    dirs = (_native.SobolDirs * (1 + replicas))(*[_native.sobol_dirs(4, base + 1000 * k)
                                                   for k in range(1 + replicas)])
    return opts, dirs


def vegas_state(device: torch.device, points: int) -> torch.Tensor:
    """A zero-filled per-parent Vegas state (no grids yet) for one evolution."""
    lib = _native.load()
    return torch.zeros(int(lib.nlo_bk_vegas_state_doubles(points, VEGAS_BINS)), dtype=torch.float64, device=device)


_workspaces: dict[tuple[int, int], torch.Tensor] = {}


def workspace(device: torch.device, points: int, vegas: _native.BKVegasOptions | None = None) -> torch.Tensor:
    """Device scratch for the right-hand side (cached per device and grid size), large
    enough for the Vegas buffers when ``vegas`` options are given."""

    lib = _native.load()
    index = device.index if device.index is not None else torch.cuda.current_device()
    key = (index, points)
    need = int(lib.nlo_bk_rhs_workspace_bytes(points))
    if vegas is not None:
        need = max(need, int(lib.nlo_bk_vegas_workspace_bytes(points, vegas)))
    buffer = _workspaces.get(key)
    if buffer is None or buffer.numel() < need:
        buffer = torch.empty(need, dtype=torch.uint8, device=torch.device("cuda", index))
        _workspaces[key] = buffer
    return buffer


def _cuda_device(device: torch.device | str) -> torch.device:
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError(
            f"device {device} is not supported: the B200 implementation runs on CUDA only (no CPU fallback)"
        )
    if not torch.cuda.is_available():
        raise RuntimeError("CUDA is not available: the B200 implementation has no CPU fallback")
    return device


def initial_row(initial_condition: MV | ICDataFile, r_host: torch.Tensor, device: torch.device) -> torch.Tensor:
    """The initial amplitude row (float64) on the device: a tabulated initial condition is
    fitted and evaluated there (nlo_ic_spline / nlo_ic_evaluate), MV is evaluated on the
    host grid (initial_conditions.py:29-35) and copied in."""
    if isinstance(initial_condition, ICDataFile):
        return initial_condition.device_amplitude(r_host.to(device=device, dtype=torch.float64))
    return initial_condition.dipole_amplitude(r_host.to(torch.float64)).to(torch.float64).to(device)


def _steps_to(y_start: float, maxy: float, step: float) -> list[float]:
    """Rapidities after each step, as bk/evolution.py:108-159 accumulates them."""

    ys = []
    y = y_start
    while True:
        y = y + step
        ys.append(y)
        if y >= maxy - 1e-12 * max(1.0, abs(maxy), abs(step)):
            break
    return ys


def rhs(
    N: torch.Tensor,
    r: torch.Tensor,
    config: BKConfig = BKConfig(),
    *,
    seed: int | None = None,
    precision: int | None = None,
    history: tuple[torch.Tensor, torch.Tensor] | None = None,
    vegas_grids: torch.Tensor | None = None,
) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """dN/dY, K1 and K2+Kf (each [R] float64) for one amplitude row (bk/evolution.py:329-488).

    ``history`` = (y [rows], N [rows, R]) is the amplitude history the kinematical
    constraint reads (its last row the current amplitude; _derivative_components'
    rapidity, history_y, history_N).  With IntegrationMethod.VEGAS, ``vegas_grids`` (from
    ``vegas_state``) carries the parents' grids from call to call; without it every call
    starts from uniform grids, as the reference does without vegas_states."""

    device = _cuda_device(r.device)
    r64 = r.to(device=device, dtype=torch.float64).contiguous()
    N64 = N.to(device=device, dtype=torch.float64).contiguous()
    points = r64.numel()
    prec = precision if precision is not None else precision_of(config, r.dtype)
    params = params_of(config, prec)
    lower, width = nlo_box(float(r64[0]), float(r64[-1]))
    dirs = _native.sobol_dirs(4, 0 if seed is None else seed)
    box = _native.box(lower, width)
    dndy = torch.empty_like(N64)
    k1 = torch.empty_like(N64)
    k2kf = torch.empty_like(N64)
    opts = vegas_options_of(config)
    ws = workspace(device, points, opts)
    lib = _native.load()
    if opts is not None:
        if config.KINEMATICAL_CONSTRAINT:
            if history is None:
                raise ValueError("kinematical evolution requires rapidity and amplitude history")
            hist_y = history[0].to(device=device, dtype=torch.float64).contiguous()
            hist_N = history[1].to(device=device, dtype=torch.float64).contiguous()
            if hist_N.ndim != 2 or hist_N.shape[1] != points or hist_y.numel() != hist_N.shape[0]:
                raise ValueError("history must be (y [rows], N [rows, points])")
        else:
            hist_y, hist_N = None, N64.unsqueeze(0)
        grids = vegas_grids if vegas_grids is not None else vegas_state(device, points)
        with torch.cuda.device(device):
            _native.check(
                lib.nlo_bk_rhs_vegas(
                    params, r64.data_ptr(), points, None if hist_y is None else hist_y.data_ptr(), hist_N.data_ptr(),
                    hist_N.shape[0], 0, 1, opts, dirs, box, grids.data_ptr(), dndy.data_ptr(), k1.data_ptr(),
                    k2kf.data_ptr(), ws.data_ptr(), ws.numel(), _native.stream_handle(device),
                )
            )
        return dndy, k1, k2kf
    if config.KINEMATICAL_CONSTRAINT:
        if history is None:
            raise ValueError("kinematical evolution requires rapidity and amplitude history")
        hist_y = history[0].to(device=device, dtype=torch.float64).contiguous()
        hist_N = history[1].to(device=device, dtype=torch.float64).contiguous()
        if hist_N.ndim != 2 or hist_N.shape[1] != points or hist_y.numel() != hist_N.shape[0]:
            raise ValueError("history must be (y [rows], N [rows, points])")
        with torch.cuda.device(device):
            _native.check(
                lib.nlo_bk_rhs_history(
                    params, r64.data_ptr(), points, hist_y.data_ptr(), hist_N.data_ptr(), hist_N.shape[0], dirs,
                    int(config.MCINTPOINTS), box, dndy.data_ptr(), k1.data_ptr(), k2kf.data_ptr(), ws.data_ptr(),
                    ws.numel(), _native.stream_handle(device),
                )
            )
        return dndy, k1, k2kf
    with torch.cuda.device(device):
        _native.check(
            lib.nlo_bk_rhs(
                params, r64.data_ptr(), N64.data_ptr(), points, dirs, int(config.MCINTPOINTS), box,
                dndy.data_ptr(), k1.data_ptr(), k2kf.data_ptr(), ws.data_ptr(), ws.numel(),
                _native.stream_handle(device),
            )
        )
    return dndy, k1, k2kf


class AdaptiveRK2:
    """The adaptive RK2 stepper of the reference (_adaptive_rk2_to, bk/evolution.py:239-326;
    its stepper off the CUDA float32 path) over the device right-hand side: a midpoint step
    of size h against two of size h/2, the error |two halves - one step|/3 against
    DE_SOLVER_ABSERR + DE_SOLVER_RELERR |two halves|, accepted when the largest ratio is at
    most 1 -- h then grows by min(5, 0.9 ratio^(-1/3)), by 5 for a zero error -- else retried
    with h shrunk by max(0.1, 0.9 ratio^(-1/3)).  ``h`` carries over from one output step to
    the next.  Each attempt reads its error ratio back to the host; the stage combinations
    run in nlo_bk_stage.  A retried attempt reuses the right-hand side at its starting row,
    which does not change with h (same row, same points)."""

    def __init__(self, config: BKConfig, r64: torch.Tensor, seed: int | None, precision: int):
        self.config, self.r64, self.seed, self.precision = config, r64, seed, precision
        self.h = float(config.DE_SOLVER_STEP)
        self.eps = float(torch.finfo(torch.float32 if precision == _native.PRECISION_MIXED else torch.float64).eps)
        self.lib = _native.load()
        self.stream = _native.stream_handle(r64.device)

    def _f(self, N: torch.Tensor) -> torch.Tensor:
        return rhs(N, self.r64, self.config, seed=self.seed, precision=self.precision)[0]

    def _stage(self, N: torch.Tensor, k: torch.Tensor, c: float) -> torch.Tensor:
        out = torch.empty_like(N)
        kp = (ctypes.c_void_p * 1)(k.data_ptr())
        cf = (ctypes.c_double * 1)(c)
        _native.check(self.lib.nlo_bk_stage(N.data_ptr(), kp, cf, 1, N.numel(), 0, out.data_ptr(), None,
                                            self.stream))
        return out

    def advance(self, N: torch.Tensor, y: float, nexty: float) -> tuple[torch.Tensor, float]:
        """(N, y) at the end of the accepted steps from y to nexty."""
        cfg = self.config
        k1 = None
        with torch.cuda.device(self.r64.device):
            while y < nexty:
                step = min(self.h, nexty - y)
                if k1 is None:
                    k1 = self._f(N)
                full = self._stage(N, self._f(self._stage(N, k1, 0.5 * step)), step)
                half_step = step / 2
                half = self._stage(N, self._f(self._stage(N, k1, 0.5 * half_step)), half_step)
                k1h = self._f(half)
                two = self._stage(half, self._f(self._stage(half, k1h, 0.5 * half_step)), half_step)
                error = torch.abs(two - full) / 3
                tolerance = cfg.DE_SOLVER_ABSERR + cfg.DE_SOLVER_RELERR * torch.abs(two)
                ratio = float(torch.max(error / tolerance).item())
                if ratio <= 1:
                    N = two
                    y += step
                    k1 = None
                    self.h = step * (5.0 if ratio == 0 else min(5.0, 0.9 * ratio ** (-1 / 3)))
                else:
                    self.h = step * max(0.1, 0.9 * ratio ** (-1 / 3))
                    if self.h <= self.eps * max(1.0, abs(y)):
                        raise RuntimeError(f"BK RK2 step underflow at y={y}")
        return N, y

    def rows(self, N0: torch.Tensor, steps: int) -> torch.Tensor:
        """Rows [steps+1, R] of output steps of DE_SOLVER_STEP from N0 (clamped to [0, 1] after
        each when FORCE_POSITIVE_N; a non-finite row raises FloatingPointError)."""
        rows = [N0]
        N, y = N0, 0.0
        for _ in range(steps):
            N, y = self.advance(N, y, y + float(self.config.DE_SOLVER_STEP))
            if self.config.FORCE_POSITIVE_N:
                N = N.clamp(0.0, 1.0)
            if not bool(torch.isfinite(N).all()):
                raise FloatingPointError(f"non-finite BK amplitude after rapidity step y={y}")
            rows.append(N)
        return torch.stack(rows)


def _evolve_rows(
    N0: torch.Tensor,
    r64: torch.Tensor,
    steps: int,
    config: BKConfig,
    seed: int | None,
    precision: int,
    *,
    history_N: torch.Tensor | None = None,
    y_all: list[float] | None = None,
    vegas_grids: torch.Tensor | None = None,
) -> torch.Tensor:
    """Rows [steps+1, R] from N0.  With the kinematical constraint the evolution reads
    the history: ``history_N`` the rows before N0 (may be empty) and ``y_all`` the
    rapidities of history, N0 and every new row.  ``vegas_grids`` (IntegrationMethod.VEGAS)
    holds the parents' grids; a fresh buffer is used when it is None."""
    device = r64.device
    if config.stepper == "rk2_adaptive":
        return AdaptiveRK2(config, r64, seed, precision).rows(N0.to(torch.float64), steps)
    points = r64.numel()
    status = torch.zeros(1, dtype=torch.int32, device=device)
    params = params_of(config, precision)
    lower, width = nlo_box(float(r64[0]), float(r64[-1]))
    box = _native.box(lower, width)
    opts, dirs_all = vegas_evolution_setup(config, seed)
    dirs = dirs_all[0]
    ws = workspace(device, points, opts)
    lib = _native.load()
    if opts is not None:
        kc = bool(config.KINEMATICAL_CONSTRAINT)
        before = 0 if (history_N is None or not kc) else history_N.shape[0]
        table = torch.empty((before + steps + 1, points), dtype=torch.float64, device=device)
        if before:
            table[:before] = history_N.to(device=device, dtype=torch.float64)
        table[before] = N0
        if kc:
            if y_all is None or len(y_all) != before + steps + 1:
                raise ValueError("kinematical evolution requires the rapidities of every row")
            y = torch.tensor(y_all, dtype=torch.float64, device=device)
        grids = vegas_grids if vegas_grids is not None else vegas_state(device, points)
        with torch.cuda.device(device):
            _native.check(
                lib.nlo_bk_evolve_vegas(
                    params, r64.data_ptr(), points, y.data_ptr() if kc else None, before, steps,
                    float(config.DE_SOLVER_STEP), _native.STEPPERS[config.stepper], opts, dirs_all, box,
                    grids.data_ptr(), table.data_ptr(), status.data_ptr(), ws.data_ptr(), ws.numel(),
                    _native.stream_handle(device),
                )
            )
        if int(status.item()) != 0:
            raise FloatingPointError("non-finite BK amplitude during the rapidity evolution")
        return table[before:]
    if config.KINEMATICAL_CONSTRAINT:
        before = 0 if history_N is None else history_N.shape[0]
        if y_all is None or len(y_all) != before + steps + 1:
            raise ValueError("kinematical evolution requires the rapidities of every row")
        table = torch.empty((before + steps + 1, points), dtype=torch.float64, device=device)
        if before:
            table[:before] = history_N.to(device=device, dtype=torch.float64)
        table[before] = N0
        y = torch.tensor(y_all, dtype=torch.float64, device=device)
        with torch.cuda.device(device):
            _native.check(
                lib.nlo_bk_evolve_history(
                    params, r64.data_ptr(), points, y.data_ptr(), before, steps, float(config.DE_SOLVER_STEP),
                    _native.STEPPERS[config.stepper], dirs, int(config.MCINTPOINTS), box, table.data_ptr(),
                    status.data_ptr(), ws.data_ptr(), ws.numel(), _native.stream_handle(device),
                )
            )
        if int(status.item()) != 0:
            raise FloatingPointError("non-finite BK amplitude during the rapidity evolution")
        return table[before:]
    table = torch.empty((steps + 1, points), dtype=torch.float64, device=device)
    table[0] = N0
    with torch.cuda.device(device):
        _native.check(
            lib.nlo_bk_evolve(
                params, r64.data_ptr(), points, steps, float(config.DE_SOLVER_STEP),
                _native.STEPPERS[config.stepper], dirs, int(config.MCINTPOINTS), box, table.data_ptr(),
                status.data_ptr(), ws.data_ptr(), ws.numel(), _native.stream_handle(device),
            )
        )
    if int(status.item()) != 0:
        raise FloatingPointError("non-finite BK amplitude during the rapidity evolution")
    return table


def solve_bk(
    initial_condition: MV | ICDataFile,
    maxy: float,
    config: BKConfig = BKConfig(),
    *,
    device: torch.device | str = "cuda",
    dtype: torch.dtype = torch.float32,
    seed: int | None = None,
) -> DipoleTable:
    """Evolve the initial condition through full steps of DE_SOLVER_STEP up to maxy
    and return the table (bk/evolution.py:33-58)."""

    if isinstance(initial_condition, ICDataFile):
        device = initial_condition.r.device if initial_condition.r.is_cuda else device
        dtype = initial_condition.r.dtype
    device = _cuda_device(device)
    # the grid and the initial row are formed on the host in float64 and copied in
    r_host = _r_grid(config, device="cpu", dtype=torch.float64)
    r64 = r_host.to(device, non_blocking=True)
    if isinstance(initial_condition, ICDataFile):
        N0 = initial_condition.device_amplitude(r64)  # the tabulated IC's spline on the device
    else:
        N0 = initial_condition.dipole_amplitude(r_host).to(torch.float64).to(device, non_blocking=True)
    ys = _steps_to(0.0, maxy, config.DE_SOLVER_STEP)
    table = _evolve_rows(N0, r64, len(ys), config, seed, precision_of(config, dtype), y_all=[0.0, *ys])
    y = torch.tensor([0.0, *ys], dtype=dtype, device=device)
    return DipoleTable(r=r64.to(dtype), y=y, N=table.to(dtype), x0=initial_condition.x0)


def evolve_table(
    table: DipoleTable,
    maxy: float,
    config: BKConfig = BKConfig(),
    *,
    seed: int | None = None,
    vegas_grids: torch.Tensor | None = None,
) -> DipoleTable:
    """Continue an existing table (e.g. one read by load_bk_table) from its last row:
    the resume path of bk/evolution.py:85-96.  With IntegrationMethod.VEGAS the parents'
    grids start uniform unless ``vegas_grids`` (``vegas_state``) carries earlier ones."""

    device = _cuda_device(table.r.device)
    r64 = table.r.to(torch.float64)
    start = float(table.y[-1].item())
    ys = _steps_to(start, maxy, config.DE_SOLVER_STEP)
    history = table.N[:-1] if config.KINEMATICAL_CONSTRAINT else None
    rows = _evolve_rows(table.N[-1].to(torch.float64), r64, len(ys), config, seed,
                        precision_of(config, table.r.dtype), history_N=history,
                        y_all=[float(v) for v in table.y.double().tolist()] + list(ys), vegas_grids=vegas_grids)
    y = torch.cat((table.y, torch.tensor(ys, dtype=table.y.dtype, device=device)))
    N = torch.cat((table.N, rows[1:].to(table.N.dtype)), dim=0)
    return DipoleTable(r=table.r, y=y, N=N, x0=table.x0)


def bk_steps(table: DipoleTable, maxy: float, config: BKConfig = BKConfig(), *,
             seed: int | None = None) -> Iterator[DipoleTable]:
    """Yield the growing table after every step (the generator of bk/evolution.py:85-159);
    the Vegas grids of the parents carry over from step to step as in the reference."""

    current = table
    if config.stepper == "rk2_adaptive":  # one stepper for the whole generator: h carries over
        device = _cuda_device(table.r.device)
        stepper = AdaptiveRK2(config, table.r.to(torch.float64), seed, precision_of(config, table.r.dtype))
        N, y0 = current.N[-1].to(torch.float64), float(current.y[-1].item())
        for y in _steps_to(y0, maxy, config.DE_SOLVER_STEP):
            N, _ = stepper.advance(N, y0, y)
            y0 = y
            if config.FORCE_POSITIVE_N:
                N = N.clamp(0.0, 1.0)
            if not bool(torch.isfinite(N).all()):
                raise FloatingPointError(f"non-finite BK amplitude after rapidity step y={y}")
            current = DipoleTable(r=current.r, y=torch.cat((current.y, torch.tensor([y], dtype=current.y.dtype,
                                                                                    device=device))),
                                  N=torch.cat((current.N, N.to(current.N.dtype).unsqueeze(0)), dim=0), x0=current.x0)
            yield current
        return
    grids = vegas_state(_cuda_device(table.r.device), table.r.numel()) \
        if config.INTMETHOD_NLO is IntegrationMethod.VEGAS else None
    for y in _steps_to(float(table.y[-1].item()), maxy, config.DE_SOLVER_STEP):
        current = evolve_table(current, y, config, seed=seed, vegas_grids=grids)
        yield current


def compute_dndy(
    initial_condition: MV | ICDataFile,
    config: BKConfig = BKConfig(),
    *,
    device: torch.device | str = "cuda",
    dtype: torch.dtype = torch.float32,
    seed: int | None = None,
) -> DNDYResult:
    """K1 and K2+Kf at the initial rapidity for the active parents (bk/evolution.py:61-82)."""

    if isinstance(initial_condition, ICDataFile):
        device = initial_condition.r.device if initial_condition.r.is_cuda else device
        dtype = initial_condition.r.dtype
    device = _cuda_device(device)
    r64 = _r_grid(config, device=device, dtype=torch.float64)
    if isinstance(initial_condition, ICDataFile):
        N = initial_condition.device_amplitude(r64)
    else:
        N = initial_condition.dipole_amplitude(r64).to(torch.float64)
    # the history of the initial rapidity alone (bk/evolution.py:76-79)
    history = (torch.zeros(1, dtype=torch.float64, device=device), N.unsqueeze(0))
    _, K1, K2_Kf = rhs(N, r64, config, seed=seed, precision=precision_of(config, dtype), history=history)
    keep = (torch.arange(r64.numel(), device=device) > 0) & (N <= 0.99999)
    return DNDYResult(r=r64[keep].to(dtype), K1=K1[keep].to(dtype), K2_Kf=K2_Kf[keep].to(dtype),
                      N=N[keep].to(dtype))


__all__ = ["AdaptiveRK2", "DNDYResult", "bk_steps", "compute_dndy", "evolve_table", "nlo_box", "rhs", "solve_bk",
           "vegas_evolution_setup", "vegas_options_of", "vegas_state"]
