"""Fixed-Sobol integration of the qqbar-g cross section (interface of the reference's
dis/fixed_sobol.py:1-381), with the whole flow -- grid training on I1/I2/I3 scores,
frozen-grid replicates -- in one device call (``nlo_dis_fixed_sobol``).

``gbw_qg_fixed_sobol`` is the fast path ``sigma_qg_d2b`` takes for the GBW dipole, as in
the reference; the device entry point also accepts a BK table.  The generic helpers
(``make_sobol_points``, ``map_importance_grid``, ``paired_endpoint_inputs``,
``learn_triple_importance_grid``, ``integrate_triple_fixed_sobol``) keep the reference's
signatures for callers that drive their own integrands; they run on device tensors.
"""

from __future__ import annotations

import ctypes
import math
from collections.abc import Callable
from dataclasses import dataclass

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.dipole.amplitude import GBW, BKDipole
from nlo_bk_optimized_b200.dis.config import DISConfig, Polarization, Quark
from nlo_bk_optimized_b200.numerics.integration import IntegralResult, sobol_dirs_array

TRAINING_SAMPLES = 65_536
TRAINING_ROUNDS = 3
SAMPLES_PER_REPLICATE = 32_768
REPLICATES = 7
GRID_BINS = 32
FIXED_SOBOL_EVALUATIONS = 2 * (TRAINING_ROUNDS * TRAINING_SAMPLES + REPLICATES * SAMPLES_PER_REPLICATE)

TripleIntegrand = Callable[[torch.Tensor], tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]]
I1SumIntegrand = Callable[[torch.Tensor, torch.Tensor], tuple[torch.Tensor, torch.Tensor]]
NestedIntegrand = Callable[[torch.Tensor], tuple[torch.Tensor, torch.Tensor]]


@dataclass(frozen=True, slots=True)
class SobolPointSet:
    training: tuple[torch.Tensor, ...]
    replicates: tuple[torch.Tensor, ...]
    seed: int


@dataclass(frozen=True, slots=True)
class FixedSobolResult:
    contributions: tuple[IntegralResult, IntegralResult, IntegralResult]
    total: IntegralResult


def make_sobol_points(dimensions: int, *, training_samples: int, training_rounds: int, samples_per_replicate: int,
                      replicates: int, device: torch.device, dtype: torch.dtype, seed: int) -> SobolPointSet:
    """Independently scrambled Sobol point sets (seeds seed + r and seed + 10000 + j),
    drawn on the device bit-exactly to SobolEngine.draw_base2 (dis/fixed_sobol.py:66-97)."""
    from nlo_bk_optimized_b200.kernels import sobol_draw

    if dimensions < 1 or training_rounds < 1 or replicates < 2:
        raise ValueError("dimensions and training rounds must be positive; replicates must exceed one")
    for count in (training_samples, samples_per_replicate):
        if count < 2 or count & (count - 1):
            raise ValueError("Sobol sample counts must be powers of two greater than one")
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError("the device Sobol generator needs a CUDA device")
    training = tuple(sobol_draw(dimensions, seed + r, training_samples, dtype=dtype, device=device)
                     for r in range(training_rounds))
    estimates = tuple(sobol_draw(dimensions, seed + 10_000 + j, samples_per_replicate, dtype=dtype, device=device)
                      for j in range(replicates))
    return SobolPointSet(training, estimates, seed)


def map_importance_grid(points: torch.Tensor, edges: torch.Tensor):
    bins = edges.shape[1] - 1
    scaled = points * bins
    bin_index = scaled.floor().to(torch.long).clamp_max(bins - 1)
    fraction = scaled - bin_index
    left = torch.gather(edges, 1, bin_index.T).T
    right = torch.gather(edges, 1, (bin_index + 1).T).T
    width = right - left
    return (left + width * fraction).contiguous(), torch.prod(bins * width, dim=1), bin_index


def paired_endpoint_inputs(source: torch.Tensor, maxr: float, *, fold_angle: bool = False):
    parent = maxr * source[:, 2]
    radial = source[:, 3]
    af = 0.5 * source[:, 4] if fold_angle else source[:, 4]
    angle = 2 * torch.pi * af
    c, s = torch.cos(angle), torch.sin(angle)
    tiny = torch.finfo(source.dtype).tiny
    closer = torch.where(c > 0, parent / (2 * c.clamp_min(tiny)), torch.full_like(parent, torch.inf))
    first_limit = torch.minimum(torch.full_like(parent, maxr), closer)
    first = source.clone()
    first[:, 3] = radial * first_limit / maxr
    first[:, 4] = af
    disk = parent * c + torch.sqrt((maxr**2 - parent.square() * s.square()).clamp_min(0))
    second_limit = torch.minimum(disk, closer).clamp_min(0)
    sr = radial * second_limit
    gx, gy = parent - sr * c, sr * s
    gr = torch.sqrt(gx.square() + gy.square())
    second = source.clone()
    second[:, 3] = gr / maxr
    second[:, 4] = torch.atan2(gy, gx).remainder(2 * torch.pi) / (2 * torch.pi)
    return first.contiguous(), first_limit / maxr, second.contiguous(), sr * second_limit / (gr.clamp_min(tiny) * maxr)


def _adapt(edges: torch.Tensor, histogram: torch.Tensor, count: torch.Tensor) -> torch.Tensor:
    bins = histogram.shape[1]
    imp = histogram / count.clamp_min(1)
    sm = imp.clone()
    sm[:, 1:-1] = (imp[:, :-2] + imp[:, 1:-1] + imp[:, 2:]) / 3
    sm[:, 0] = (imp[:, 0] + imp[:, 1]) / 2
    sm[:, -1] = (imp[:, -2] + imp[:, -1]) / 2
    sm = sm + torch.finfo(edges.dtype).eps
    rows = []
    for d in range(histogram.shape[0]):
        cum = torch.cat((edges.new_zeros(1), torch.cumsum(sm[d], dim=0)))
        target = torch.linspace(0, float(cum[-1]), bins + 1, dtype=edges.dtype, device=edges.device)
        idx = torch.searchsorted(cum, target, right=True).sub(1).clamp(0, bins - 1)
        frac = (target - cum[idx]) / sm[d, idx]
        row = edges[d, idx] + frac * (edges[d, idx + 1] - edges[d, idx])
        row[0], row[-1] = 0, 1
        rows.append(row)
    return torch.stack(rows)


@torch.no_grad()
def learn_triple_importance_grid(function: TripleIntegrand, training_points: tuple[torch.Tensor, ...], *,
                                 maxr: float, bins: int = GRID_BINS, fold_angle: bool = True,
                                 i1_weight: float = 1.0) -> torch.Tensor:
    """One frozen grid from normalised I1, I2, I3 magnitudes (dis/fixed_sobol.py:161-211)."""
    if not training_points:
        raise ValueError("at least one independent training point set is required")
    ref = training_points[0]
    dims = ref.shape[1]
    edges = torch.linspace(0, 1, bins + 1, device=ref.device, dtype=ref.dtype).expand(dims, -1).clone()
    for points in training_points:
        source, inv, bi = map_importance_grid(points, edges)
        first, fw, second, sw = paired_endpoint_inputs(source, maxr, fold_angle=fold_angle)
        a_reg, a_sens, a2, a3 = function(first)
        b_reg, b_sens, b2, b3 = function(second)
        weighted = tuple((f * fw + s * sw) * inv for f, s in zip((a_reg + a_sens.to(a_reg.dtype), a2, a3),
                                                                (b_reg + b_sens.to(b_reg.dtype), b2, b3)))
        tiny = torch.finfo(ref.dtype).tiny
        score = sum(w * v.abs() / v.abs().mean().clamp_min(tiny) for w, v in zip((i1_weight, 1.0, 1.0), weighted))
        hist = ref.new_zeros((dims, bins))
        count = ref.new_zeros((dims, bins))
        for d in range(dims):
            hist[d].scatter_add_(0, bi[:, d], score.to(ref.dtype))
            count[d].scatter_add_(0, bi[:, d], torch.ones_like(score, dtype=ref.dtype))
        edges = _adapt(edges, hist, count)
    return edges


def _replicate_result(values: torch.Tensor, samples: int, epsrel: float, seed: int) -> IntegralResult:
    value = values.mean()
    error = values.std(unbiased=True) / math.sqrt(values.numel())
    return IntegralResult(value, error, samples, bool(error <= epsrel * value.abs()), seed)


@torch.no_grad()
def integrate_triple_fixed_sobol(i1_sum_function: I1SumIntegrand, nested_function: NestedIntegrand,
                                 edges: torch.Tensor, replicate_points: tuple[torch.Tensor, ...], *, maxr: float,
                                 epsrel: float, seed: int, training_evaluations: int = 0) -> FixedSobolResult:
    """I1, I2, I3 and their correlated sum from frozen-grid replicates
    (dis/fixed_sobol.py:214-270)."""
    if len(replicate_points) < 2:
        raise ValueError("at least two scrambled Sobol replicates are required")
    estimates = []
    for points in replicate_points:
        if edges.numel():
            source, inv, _ = map_importance_grid(points, edges)
            first, fw, second, sw = paired_endpoint_inputs(source, maxr, fold_angle=True)
            fw, sw = fw * inv, sw * inv
        else:
            first, fw, second, sw = points, torch.ones(points.shape[0]), points, torch.zeros(points.shape[0])
        r1, s1 = i1_sum_function(first, fw)
        r2, s2 = i1_sum_function(second, sw)
        f2, f3 = nested_function(first)
        g2, g3 = nested_function(second)
        n = points.shape[0]
        i1 = (r1.sum() + r2.sum()) / n + ((s1.sum() + s2.sum()) / n).to(r1.dtype)
        estimates.append(torch.stack((i1.double(), (f2 * fw + g2 * sw).double().mean(),
                                      (f3 * fw + g3 * sw).double().mean())))
    stacked = torch.stack(estimates)
    samples = training_evaluations + 2 * sum(p.shape[0] for p in replicate_points)
    parts = tuple(_replicate_result(stacked[:, k], samples, epsrel, seed) for k in range(3))
    return FixedSobolResult(parts, _replicate_result(stacked.sum(dim=1), samples, epsrel, seed))


def fixed_sobol_device(Q2: float, xbj: float, polarization: Polarization, quark: Quark, dipole: GBW | BKDipole,
                       config: DISConfig, *, seed: int, device: torch.device, precision: int,
                       training_samples: int = TRAINING_SAMPLES, training_rounds: int = TRAINING_ROUNDS,
                       samples_per_replicate: int = SAMPLES_PER_REPLICATE, replicates: int = REPLICATES,
                       bins: int = GRID_BINS, i1_weight: float = 1.0) -> tuple[torch.Tensor, torch.Tensor]:
    """Run nlo_dis_fixed_sobol; returns (grid state, replicate estimates [replicates, 3]) on the device."""
    from nlo_bk_optimized_b200.dis.observables import kinematics

    lib = _native.load()
    o = _native.FixedSobolOptions(training_samples=training_samples, training_rounds=training_rounds,
                                  samples_per_replicate=samples_per_replicate, replicates=replicates, bins=bins,
                                  fold_angle=1, i1_weight=i1_weight, inner_points=config.cuda_nested_points,
                                  precision=precision)
    ws_bytes = int(lib.nlo_dis_fixed_sobol_workspace_bytes(ctypes.byref(o)))
    if ws_bytes == 0:
        raise ValueError("invalid fixed-Sobol options")
    workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
    grid = torch.empty(int(lib.nlo_dis_fixed_sobol_grid_doubles(bins)), dtype=torch.float64, device=device)
    estimates = torch.empty((replicates, 3), dtype=torch.float64, device=device)
    seeds = [seed + r for r in range(training_rounds)] + [seed + 10_000 + j for j in range(replicates)]
    dirs = sobol_dirs_array(5, seeds)
    kin = kinematics(Q2, xbj, polarization, config, quark)
    with torch.cuda.device(device):
        _native.check(lib.nlo_dis_fixed_sobol(ctypes.byref(kin), ctypes.byref(dipole.native()), ctypes.byref(o), dirs,
                                              grid.data_ptr(), estimates.data_ptr(), workspace.data_ptr(), ws_bytes,
                                              _native.stream_handle(device)))
    return grid, estimates


def gbw_qg_fixed_sobol(Q2: torch.Tensor, xbj: torch.Tensor, polarization: Polarization, quark: Quark, dipole: GBW,
                       config: DISConfig, *, seed: int) -> FixedSobolResult:
    """One quark's complete qqbar-g contribution by the fixed-Sobol path
    (dis/fixed_sobol.py:273-368); mixed precision for float32 Q2, FP64 for float64."""
    if Q2.numel() != 1 or xbj.numel() != 1:
        raise ValueError("fixed-Sobol DIS requires scalar Q2 and xbj")
    device = Q2.device if Q2.is_cuda else torch.device("cuda", torch.cuda.current_device())
    precision = _native.PRECISION_FP64 if Q2.dtype == torch.float64 else _native.PRECISION_MIXED
    _, est = fixed_sobol_device(float(Q2), float(xbj), polarization, quark, dipole, config, seed=seed,
                                device=device, precision=precision)
    est = est.cpu()
    samples = FIXED_SOBOL_EVALUATIONS
    parts = tuple(_replicate_result(est[:, k], samples, config.epsrel, seed) for k in range(3))
    total = _replicate_result(est.sum(dim=1), samples, config.epsrel, seed)
    to = lambda r: IntegralResult(r.value.to(device), r.error.to(device), r.n_eval, r.converged, r.seed)  # noqa: E731
    return FixedSobolResult(tuple(to(r) for r in parts), to(total))


__all__ = [
    "FIXED_SOBOL_EVALUATIONS",
    "FixedSobolResult",
    "SobolPointSet",
    "fixed_sobol_device",
    "gbw_qg_fixed_sobol",
    "integrate_triple_fixed_sobol",
    "learn_triple_importance_grid",
    "make_sobol_points",
    "map_importance_grid",
    "paired_endpoint_inputs",
]
