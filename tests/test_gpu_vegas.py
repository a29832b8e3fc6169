"""The general vegas() integrator (numerics/integration.py:120-589 of the reference) on the
device: the reference's own grid-reuse test, the oracle's Vegas driver on the same Sobol
points, and known integrals."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

import oracle
from nlo_bk_optimized_b200.numerics import VegasState, vegas
from oracle import dis as odis

pytestmark = pytest.mark.gpu


def test_vegas_reuses_grid_with_quarter_warmup():
    """The reference's test_vegas_reuses_grid_with_quarter_warmup
    (tests/test_bk_production.py:52-74) on a CUDA box."""
    bounds = torch.tensor([[0.0, 1.0], [0.0, 1.0]], dtype=torch.float64, device="cuda")
    state = VegasState()
    arguments = {
        "samples_per_iteration": 2_000,
        "warmup_samples": 400,
        "max_iterations": 2,
        "min_iterations": 2,
        "epsrel": 1.0,
        "seed": 73,
        "state": state,
        "reuse_warmup_fraction": 0.25,
    }
    first = vegas(lambda x: x[:, 0].square() + x[:, 1], bounds, **arguments)
    assert first.n_eval == 4_400
    assert state.edges is not None
    first_edges = state.edges.clone()
    second = vegas(lambda x: x[:, 0].square() + x[:, 1], bounds, **arguments)
    assert second.n_eval == 4_100
    assert state.edges is not None
    assert not torch.equal(state.edges, first_edges)
    for result in (first, second):
        assert abs(float(result.value) - 5.0 / 6.0) < 5 * float(result.error) + 1e-3


def test_vegas_matches_the_oracle_driver_on_the_same_points():
    dims, bins, seed = 3, 16, 5
    samples, warm, iterations = 3000, 600, 4
    bounds = torch.tensor([[0.0, 1.0]] * dims, dtype=torch.float64, device="cuda")

    def f_torch(x):
        return torch.exp(-8.0 * ((x - 0.3) ** 2).sum(dim=1)) + 0.1 * x[:, 0]

    def f_numpy(x):
        return np.exp(-8.0 * ((x - 0.3) ** 2).sum(axis=1)) + 0.1 * x[:, 0]

    got = vegas(f_torch, bounds, samples_per_iteration=samples, warmup_samples=warm, max_iterations=iterations,
                min_iterations=iterations, bins=bins, epsrel=0.0, seed=seed, batch_size=1024)
    state, shift = oracle.sobol_state(dims, seed)
    offsets = [0]

    def sampler(it, n):
        u = oracle.sobol(state, shift, offsets[0], n, as_f32=False)
        offsets[0] += n
        scaled = u * bins
        bi = np.minimum(np.floor(scaled).astype(np.int64), bins - 1)
        return bi, scaled - bi

    value, error, n_eval, converged, edges = odis.vegas(f_numpy, dims, sampler, samples=samples,
                                                        max_iterations=iterations, min_iterations=iterations,
                                                        bins=bins, warmup_samples=warm, epsrel=0.0)
    assert got.n_eval == n_eval == warm + iterations * samples
    assert abs(float(got.value) - value) <= 1e-12 * abs(value)
    assert abs(float(got.error) - error) <= 1e-9 * error
    assert got.converged == converged


def test_vegas_known_integrals_and_bounds():
    # a Gaussian over a shifted box: prod over dims of int_{-1}^{2} exp(-x^2) dx
    bounds = torch.tensor([[-1.0, 2.0]] * 4, dtype=torch.float64, device="cuda")
    one = 0.5 * math.sqrt(math.pi) * (math.erf(2.0) + math.erf(1.0))
    res = vegas(lambda x: torch.exp(-(x * x).sum(dim=1)), bounds, samples_per_iteration=1 << 15, warmup_samples=4096,
                max_iterations=6, min_iterations=3, epsrel=1e-3, seed=1)
    assert abs(float(res.value) - one ** 4) < 5 * float(res.error) + 1e-4 * one ** 4
    assert res.converged and res.seed == 1
    with pytest.raises(ValueError):
        vegas(lambda x: x[:, 0], bounds, samples_per_iteration=1)
    with pytest.raises(ValueError):
        vegas(lambda x: x[:, 0], torch.tensor([[1.0, 0.0]], device="cuda", dtype=torch.float64),
              samples_per_iteration=16)
    with pytest.raises(ValueError):  # a kept grid must match the dimensions
        vegas(lambda x: x[:, 0], bounds, samples_per_iteration=16,
              state=VegasState(edges=torch.linspace(0, 1, 33, device="cuda", dtype=torch.float64).expand(2, -1)))
