"""Integration results and the device Vegas / Gauss-Legendre drivers of the DIS terms
(interface of the reference's numerics/integration.py:12-138).

``vegas_terms`` integrates one DIS term for many kinematic points in a single sequence
of device launches (libnlo_b200.so ``nlo_dis_vegas``): every Vegas iteration -- Sobol
sampling through the grid, the integrand, the |w| histograms, the grid re-binning and the
inverse-variance combination -- runs on the GPU, and the host reads the results once at
the end.  ``gauss_legendre_terms`` does the same for the tensor rule of the 2D terms.
"""

from __future__ import annotations

import ctypes
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


def vegas_terms(term: int, kins: list[_native.DisKinematics], dipole: _native.Dipole, options: VegasOptions,
                seeds: list[int], *, precision: int, device: torch.device,
                edges: torch.Tensor | None = None) -> torch.Tensor:
    """Run Vegas for len(kins) integrals of one term; returns the device state
    [jobs, state_doubles] (edges followed by value, error, n_eval, iterations, converged)."""
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


def gauss_legendre_terms(term: int, kins: list[_native.DisKinematics], dipole: _native.Dipole, points: int, *,
                         precision: int, device: torch.device) -> torch.Tensor:
    """Tensor Gauss-Legendre of a 2D term for len(kins) points: [jobs, 2] = (value, error)."""
    lib = _native.load()
    jobs = len(kins)
    out = torch.empty((jobs, 2), dtype=torch.float64, device=device)
    ws_bytes = int(lib.nlo_dis_gauss_legendre_workspace_bytes(jobs))
    workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
    karr = kinematics_array(kins)
    with torch.cuda.device(device):
        _native.check(lib.nlo_dis_gauss_legendre(karr, jobs, term, ctypes.byref(dipole), points, precision,
                                                 out.data_ptr(), workspace.data_ptr(), ws_bytes,
                                                 _native.stream_handle(device)))
    return out


__all__ = ["IntegralResult", "VegasOptions", "VegasState", "budget_options", "gauss_legendre_terms",
           "state_results", "vegas_terms"]
