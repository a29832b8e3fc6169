"""Integration results, the general ``vegas()`` integrator, and the device Vegas /
Gauss-Legendre drivers of the DIS terms (interface of the reference's
numerics/integration.py:12-138).

``vegas`` keeps the reference's keyword signature and semantics (warm-up round, the
inverse-variance combination, ``VegasState`` reuse with a shortened warm-up) for any
integrand written as a torch function of a CUDA batch of points; sampling, the grid map,
the |w| histograms, the re-binning and the combination run in libnlo_b200.so
(``nlo_vegas_*``), only the integrand is the caller's.

``vegas_terms`` integrates one DIS term for many kinematic points in a single sequence
of device launches (libnlo_b200.so ``nlo_dis_vegas``): every Vegas iteration -- Sobol
sampling through the grid, the integrand, the |w| histograms, the grid re-binning and the
inverse-variance combination -- runs on the GPU, and the host reads the results once at
the end.  ``gauss_legendre_terms`` does the same for the tensor rule of the 2D terms.
"""

from __future__ import annotations

import ctypes
from collections.abc import Callable
from dataclasses import dataclass
from functools import lru_cache

import torch

from nlo_bk_optimized_b200 import _native


@dataclass(frozen=True, slots=True)
class IntegralResult:
    value: torch.Tensor
    error: torch.Tensor
    n_eval: int
    converged: bool
    seed: int | None


@dataclass(slots=True)
class VegasState:
    """Importance grid carried between related Vegas integrals (edges [dims, bins+1])."""

    edges: torch.Tensor | None = None
    last_components: torch.Tensor | None = None
    last_error: float | None = None


@dataclass(frozen=True, slots=True)
class VegasOptions:
    samples_per_iteration: int
    max_iterations: int = 8
    min_iterations: int = 3
    warmup_samples: int = 0
    bins: int = 32
    epsrel: float = 0.2
    epsabs: float = 0.0
    inner_points: int = 48

    def native(self, precision: int, keep_edges: bool = False) -> _native.VegasOptions:
        if self.samples_per_iteration < 2 or self.max_iterations < 1:
            raise ValueError("Vegas requires at least two samples and one iteration")
        if self.min_iterations < 1 or self.min_iterations > self.max_iterations:
            raise ValueError("min_iterations must lie between one and max_iterations")
        if self.warmup_samples == 1 or self.warmup_samples < 0:
            raise ValueError("warmup_samples must be zero or at least two")
        o = _native.VegasOptions()
        o.bins = self.bins
        o.max_iterations = self.max_iterations
        o.min_iterations = self.min_iterations
        o.samples_per_iteration = self.samples_per_iteration
        o.warmup_samples = self.warmup_samples
        o.epsrel = self.epsrel
        o.epsabs = self.epsabs
        o.inner_points = self.inner_points
        o.precision = precision
        o.keep_edges = int(keep_edges)
        return o


def vegas(
    function: Callable[[torch.Tensor], torch.Tensor],
    bounds: torch.Tensor,
    *,
    samples_per_iteration: int,
    max_iterations: int = 8,
    min_iterations: int = 3,
    warmup_samples: int = 0,
    bins: int = 32,
    batch_size: int = 65_536,
    epsrel: float = 0.2,
    epsabs: float = 0.0,
    seed: int | None = None,
    cuda_mask_fusion: bool = False,
    cuda_weighted_function=None,
    state: VegasState | None = None,
    reuse_warmup_fraction: float = 0.0,
    validate_bounds: bool = True,
) -> IntegralResult:
    """Adaptive importance-sampled Vegas (numerics/integration.py:120-589) on the device.

    ``function`` maps a CUDA float64 batch of points [n, dims] to [n] values.  Points are
    scrambled Sobol points of ``seed`` (indices 0, 1, ... across the rounds; a random seed
    when None, as the reference draws one), each coordinate split into a grid bin and a
    fraction.  A warm-up round of ``warmup_samples`` adapts the grid only; then up to
    ``max_iterations`` rounds of ``samples_per_iteration`` are combined by inverse variance
    until, after ``min_iterations``, error <= max(epsabs, epsrel |value|).  A ``state``
    holding edges starts from them with a warm-up of max(2, warmup x reuse_warmup_fraction)
    (none when either is zero); the final grid is written back to it.  ``cuda_mask_fusion``
    is accepted for compatibility (the bookkeeping always runs in this library's kernels);
    ``cuda_weighted_function`` is the reference's hook for its own CUDA kernels and is not
    supported."""

    if cuda_weighted_function is not None:
        raise NotImplementedError("cuda_weighted_function is the reference's hook for its own CUDA kernels; pass the "
                                  "integrand as `function`")
    if bounds.ndim != 2 or bounds.shape[1] != 2 or bounds.shape[0] < 1:
        raise ValueError("bounds must have shape (dimensions, 2)")
    if not bounds.is_floating_point():
        raise TypeError("bounds must be floating point")
    if validate_bounds and (not bool(torch.isfinite(bounds).all()) or not bool((bounds[:, 1] > bounds[:, 0]).all())):
        raise ValueError("bounds must be finite with lower < upper")
    if samples_per_iteration < 2 or max_iterations < 1:
        raise ValueError("Vegas requires at least two samples and one iteration")
    if min_iterations < 1 or min_iterations > max_iterations:
        raise ValueError("min_iterations must lie between one and max_iterations")
    if warmup_samples == 1 or warmup_samples < 0:
        raise ValueError("warmup_samples must be zero or at least two")
    if not 0 <= reuse_warmup_fraction <= 1:
        raise ValueError("reuse_warmup_fraction must lie between zero and one")
    if bins < 2 or batch_size < 1:
        raise ValueError("bins and batch_size must be positive")
    device = bounds.device
    _native.require_cuda(bounds.contiguous(), "bounds")
    dims = int(bounds.shape[0])
    if dims > 8:
        raise ValueError("the device Vegas takes at most 8 dimensions")
    lib = _native.load()
    reused = state is not None and state.edges is not None
    grid = torch.empty(int(lib.nlo_vegas_state_doubles(dims, bins)), dtype=torch.float64, device=device)
    if reused:
        edges = state.edges
        if tuple(edges.shape) != (dims, bins + 1) or edges.device != device or edges.dtype is not bounds.dtype:
            raise ValueError("Vegas state must match the integration dimensions, bins, and device")
        if not bool(torch.isfinite(edges).all()) or not bool((edges[:, 1:] > edges[:, :-1]).all()):
            raise ValueError("Vegas state edges must be finite and strictly increasing")
        if not bool((edges[:, 0] == 0).all()) or not bool((edges[:, -1] == 1).all()):
            raise ValueError("Vegas state edges must span the unit interval")
        grid[: dims * (bins + 1)] = edges.reshape(-1).to(torch.float64)
    seed = torch.seed() % (1 << 31) if seed is None else seed
    dirs = _native.sobol_dirs(dims, seed)
    ws = torch.empty(int(lib.nlo_vegas_workspace_bytes(dims, bins)), dtype=torch.uint8, device=device)
    stream = _native.stream_handle(device)
    lower = (ctypes.c_double * dims)(*bounds[:, 0].double().tolist())
    width = (ctypes.c_double * dims)(*(bounds[:, 1] - bounds[:, 0]).double().tolist())
    warm = warmup_samples
    if reused:
        warm = max(2, int(warmup_samples * reuse_warmup_fraction)) if warmup_samples > 0 and reuse_warmup_fraction > 0 \
            else 0
    chunk = min(batch_size, max(warm, samples_per_iteration))
    x = torch.empty((chunk, dims), dtype=torch.float64, device=device)
    factor = torch.empty(chunk, dtype=torch.float64, device=device)
    bin_index = torch.empty((chunk, dims), dtype=torch.int32, device=device)
    base = dims * (bins + 1)
    offset = 0
    with torch.cuda.device(device):
        _native.check(lib.nlo_vegas_begin(dims, bins, int(reused), grid.data_ptr(), ws.data_ptr(), ws.numel(), stream))
        for round_index in range(max_iterations + int(warm > 0)):
            warmup_round = warm > 0 and round_index == 0
            n = warm if warmup_round else samples_per_iteration
            done = 0
            while done < n:
                count = min(chunk, n - done)
                _native.check(lib.nlo_vegas_sample(dirs, offset + done, count, dims, bins, grid.data_ptr(), lower,
                                                   width, x.data_ptr(), factor.data_ptr(), bin_index.data_ptr(),
                                                   stream))
                values = function(x[:count].to(bounds.dtype))
                if values.shape != (count,):
                    raise ValueError("Vegas integrands must return one value per sample")
                values = values.to(device=device, dtype=torch.float64).contiguous()
                _native.check(lib.nlo_vegas_accumulate(values.data_ptr(), factor.data_ptr(), bin_index.data_ptr(),
                                                       count, dims, bins, ws.data_ptr(), ws.numel(), stream))
                done += count
            offset += n
            _native.check(lib.nlo_vegas_end_round(dims, bins, grid.data_ptr(), n, int(warmup_round), min_iterations,
                                                  float(epsrel), float(epsabs), ws.data_ptr(), ws.numel(), stream))
            if not warmup_round and bool(grid[base + _native.VEGAS_CONVERGED].item()):
                break
    value = grid[base + _native.VEGAS_VALUE].to(bounds.dtype)
    error = grid[base + _native.VEGAS_ERROR].to(bounds.dtype)
    n_eval = int(grid[base + _native.VEGAS_EVALS].item())
    converged = bool(grid[base + _native.VEGAS_CONVERGED].item())
    if state is not None:
        state.edges = grid[:base].reshape(dims, bins + 1).to(bounds.dtype).clone()
        state.last_error = float(error.item())
    return IntegralResult(value, error, n_eval, converged, seed)


def budget_options(maxeval: int, epsrel: float, bins: int = 32) -> VegasOptions:
    """The iteration split of _vegas_with_budget (dis/observables.py:667-692)."""
    if maxeval < 2:
        raise ValueError("NLO integration requires maxeval >= 2")
    max_iterations = min(8, max(1, maxeval // 2))
    samples = max(2, maxeval // max_iterations)
    return VegasOptions(samples_per_iteration=samples, max_iterations=max_iterations,
                        min_iterations=min(3, max_iterations), bins=bins, epsrel=epsrel)


@lru_cache(maxsize=256)
def _dirs_bytes(dims: int, seed: int) -> bytes:
    return bytes(_native.sobol_dirs(dims, seed))


def sobol_dirs_array(dims: int, seeds: list[int]) -> ctypes.Array:
    arr = (_native.SobolDirs * len(seeds))()
    for i, seed in enumerate(seeds):
        ctypes.memmove(ctypes.byref(arr, i * ctypes.sizeof(_native.SobolDirs)), _dirs_bytes(dims, int(seed)),
                       ctypes.sizeof(_native.SobolDirs))
    return arr


def kinematics_array(kins: list[_native.DisKinematics]) -> ctypes.Array:
    arr = (_native.DisKinematics * len(kins))()
    for i, k in enumerate(kins):
        arr[i] = k
    return arr


def _dipole_array(dipoles: list[_native.Dipole]) -> ctypes.Array:
    arr = (_native.Dipole * len(dipoles))()
    for i, d in enumerate(dipoles):
        arr[i] = d
    return arr


def vegas_terms(term: int, kins: list[_native.DisKinematics], dipole: _native.Dipole | None, options: VegasOptions,
                seeds: list[int], *, precision: int, device: torch.device,
                edges: torch.Tensor | None = None, dipoles: list[_native.Dipole] | None = None) -> torch.Tensor:
    """Run Vegas for len(kins) integrals of one term; returns the device state
    [jobs, state_doubles] (edges followed by value, error, n_eval, iterations, converged).
    ``dipoles`` (one per job) replaces the common ``dipole``."""
    lib = _native.load()
    jobs = len(kins)
    dims = _native.DIS_DIMS[term]
    opts = options.native(precision, keep_edges=edges is not None)
    stride = int(lib.nlo_dis_vegas_state_doubles(term, options.bins))
    state = torch.zeros((jobs, stride), dtype=torch.float64, device=device)
    if edges is not None:
        state[:, : dims * (options.bins + 1)] = edges.reshape(1, -1).to(state)
    ws_bytes = int(lib.nlo_dis_vegas_workspace_bytes(jobs, term, ctypes.byref(opts)))
    if ws_bytes == 0:
        raise ValueError("invalid Vegas options")
    workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
    karr = kinematics_array(kins)
    darr = sobol_dirs_array(max(dims, 1), seeds)
    with torch.cuda.device(device):
        if dipoles is not None:
            if len(dipoles) != jobs:
                raise ValueError("one dipole per job is required")
            _native.check(lib.nlo_dis_vegas_dipoles(karr, jobs, term, _dipole_array(dipoles), ctypes.byref(opts),
                                                    darr, state.data_ptr(), workspace.data_ptr(), ws_bytes,
                                                    _native.stream_handle(device)))
        else:
            _native.check(lib.nlo_dis_vegas(karr, jobs, term, ctypes.byref(dipole), ctypes.byref(opts), darr,
                                            state.data_ptr(), workspace.data_ptr(), ws_bytes,
                                            _native.stream_handle(device)))
    return state


def state_results(state: torch.Tensor, term: int, bins: int) -> dict[str, torch.Tensor]:
    """Split device Vegas states into edges and (value, error, n_eval, iterations, converged)."""
    dims = _native.DIS_DIMS[term]
    base = dims * (bins + 1)
    return {
        "edges": state[:, :base].reshape(-1, dims, bins + 1),
        "value": state[:, base + _native.VEGAS_VALUE],
        "error": state[:, base + _native.VEGAS_ERROR],
        "n_eval": state[:, base + _native.VEGAS_EVALS],
        "iterations": state[:, base + _native.VEGAS_ITERATIONS],
        "converged": state[:, base + _native.VEGAS_CONVERGED],
    }


def gauss_legendre_terms(term: int, kins: list[_native.DisKinematics], dipole: _native.Dipole | None, points: int,
                         *, precision: int, device: torch.device,
                         dipoles: list[_native.Dipole] | None = None) -> torch.Tensor:
    """Tensor Gauss-Legendre of a 2D term for len(kins) points: [jobs, 2] = (value, error).
    ``dipoles`` (one per job) replaces the common ``dipole``."""
    lib = _native.load()
    jobs = len(kins)
    out = torch.empty((jobs, 2), dtype=torch.float64, device=device)
    ws_bytes = int(lib.nlo_dis_gauss_legendre_workspace_bytes(jobs))
    workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
    karr = kinematics_array(kins)
    with torch.cuda.device(device):
        if dipoles is not None:
            if len(dipoles) != jobs:
                raise ValueError("one dipole per job is required")
            _native.check(lib.nlo_dis_gauss_legendre_dipoles(karr, jobs, term, _dipole_array(dipoles), points,
                                                             precision, out.data_ptr(), workspace.data_ptr(),
                                                             ws_bytes, _native.stream_handle(device)))
        else:
            _native.check(lib.nlo_dis_gauss_legendre(karr, jobs, term, ctypes.byref(dipole), points, precision,
                                                     out.data_ptr(), workspace.data_ptr(), ws_bytes,
                                                     _native.stream_handle(device)))
    return out


__all__ = ["IntegralResult", "VegasOptions", "VegasState", "budget_options", "gauss_legendre_terms",
           "state_results", "vegas", "vegas_terms"]
