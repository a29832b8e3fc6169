"""Parity of the B200 kernels (libnlo_b200.so, called through its C ABI) with the
CPU oracle on identical inputs.

Tolerances: 1e-10 relative for the all-FP64 device build, 1e-4 relative for the
mixed build (FP32 integrands, FP64 sums), as stated for this path.  Relative
errors of per-parent integrals are measured against max(|oracle|, floor * max
|oracle|) so that parents whose integral is an accidental near-zero do not
divide by zero; the floor is 1e-3.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from nlo_bk_optimized_b200 import MV, BKConfig, compute_dndy, kernels, solve_bk
from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.bk.config import IntegrationMethod
from nlo_bk_optimized_b200.bk.evolution import _r_grid, evolve_table, rhs

pytestmark = pytest.mark.gpu

TOL = {_native.PRECISION_MIXED: 1e-4, _native.PRECISION_FP64: 1e-10}
PRECISIONS = [_native.PRECISION_MIXED, _native.PRECISION_FP64]
DEVICE = "cuda"


def _rel_err(gpu: np.ndarray, ref: np.ndarray, floor: float = 1e-3) -> float:
    scale = np.maximum(np.abs(ref), floor * np.max(np.abs(ref)) + 1e-300)
    return float(np.max(np.abs(gpu - ref) / scale))


def _setup(rpoints=99, minr=1e-6, maxr=1e2, qs=0.2, **kw):
    # the oracle integrates K2+Kf on fixed Sobol points and steps with RK4 unless told otherwise
    kw.setdefault("INTMETHOD_NLO", IntegrationMethod.SOBOL)
    kw.setdefault("STEPPER", "rk4")
    config = BKConfig(RPOINTS=rpoints, MINR=minr, MAXR=maxr, **kw)
    r = _r_grid(config, device=DEVICE, dtype=torch.float64)
    N = MV(qs0sqr=qs).dipole_amplitude(r)
    return config, r, N


def _sobol_points(n: int, seed: int, f32: bool, offset: int = 0) -> np.ndarray:
    state, shift = oracle.sobol_state(4, seed)
    return oracle.sobol(state, shift, offset, n, as_f32=f32)


# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dims", [1, 4, 8])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_device_sobol_bit_exact(dims, dtype):
    torch.set_default_dtype(torch.float32)
    engine = torch.quasirandom.SobolEngine(dims, scramble=True, seed=11)
    ref = engine.draw(3000, dtype=dtype)
    got = kernels.sobol_draw(dims, 11, 3000, dtype=dtype).cpu()
    assert torch.equal(got, ref)
    tail = kernels.sobol_draw(dims, 11, 1000, offset=2000, dtype=dtype).cpu()
    assert torch.equal(tail, ref[2000:])


def test_splines_match_oracle():
    config, r, N = _setup(rpoints=399, minr=1e-7)
    sp = kernels.splines(r, N)
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    for kind, key in ((0, "n"), (1, "s")):
        ref = oracle.loglog_spline(rn, Nn, kind)
        got = sp[key].cpu().numpy()
        np.testing.assert_allclose(sp["x"].cpu().numpy(), ref.x, rtol=1e-15, atol=0)
        for j, field in enumerate("abcd"):
            np.testing.assert_allclose(got[:, j], getattr(ref, field), rtol=1e-12, atol=1e-12)


def test_active_list_edges():
    config, r, N = _setup(rpoints=99)
    idx, count = kernels.active(N)
    expected = np.nonzero((np.arange(r.numel()) > 0) & (N.cpu().numpy() <= 0.99999))[0]
    assert int(count.item()) == expected.size
    np.testing.assert_array_equal(idx[: expected.size].cpu().numpy(), expected)
    idx, count = kernels.active(torch.ones_like(N))
    assert int(count.item()) == 0


@pytest.mark.parametrize("precision", PRECISIONS)
def test_k1_matches_oracle(precision):
    config, r, N = _setup(rpoints=99)
    got = kernels.k1(r, N, config, precision=precision).cpu().numpy()
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    active = (np.arange(rn.size) > 0) & (Nn <= 0.99999)
    ref = np.zeros_like(rn)
    ref[active] = oracle.k1_fixed(rn[active], oracle.loglog_spline(rn, Nn, 0), oracle.physics(config))
    assert np.all(got[~active] == 0.0)
    err = _rel_err(got[active], ref[active])
    assert err <= TOL[precision], f"K1 max relative error {err:.3e}"


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("samples", [1, 33, 1000, 4096])
def test_k2kf_matches_oracle(precision, samples):
    config, r, N = _setup(rpoints=99)
    got = kernels.k2kf(r, N, config, samples=samples, precision=precision).cpu().numpy()
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    f32 = precision == _native.PRECISION_MIXED
    pts = _sobol_points(samples, 0, f32)
    lower, width = oracle.nlo_box(rn)
    active = (np.arange(rn.size) > 0) & (Nn <= 0.99999)
    ref = np.zeros((rn.size, 3))
    ref[active] = oracle.k2kf_sums(rn[active], pts, lower, width, f32, oracle.loglog_spline(rn, Nn, 1),
                                   oracle.physics(config))
    assert np.all(got[~active] == 0.0)
    total_gpu = got[active, 0] + got[active, 1]
    total_ref = ref[active, 0] + ref[active, 1]
    tol = TOL[precision] if samples >= 1000 else 10 * TOL[precision]
    for name, a, b in (("K2", got[active, 0], ref[active, 0]), ("Kf", got[active, 1], ref[active, 1]),
                       ("K2+Kf", total_gpu, total_ref), ("sum w^2", got[active, 2], ref[active, 2])):
        err = _rel_err(a, b)
        assert err <= tol, f"{name} max relative error {err:.3e} (samples={samples})"


@pytest.mark.parametrize("precision", PRECISIONS)
def test_k2kf_large_grid_matches_oracle(precision):
    config, r, N = _setup(rpoints=399, minr=1e-7, qs=0.6)
    samples = 1 << 13
    got = kernels.k2kf(r, N, config, samples=samples, precision=precision).cpu().numpy()
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    f32 = precision == _native.PRECISION_MIXED
    active = (np.arange(rn.size) > 0) & (Nn <= 0.99999)
    lower, width = oracle.nlo_box(rn)
    ref = oracle.k2kf_sums(rn[active], _sobol_points(samples, 0, f32), lower, width, f32,
                           oracle.loglog_spline(rn, Nn, 1), oracle.physics(config))
    err = _rel_err(got[active, 0] + got[active, 1], ref[:, 0] + ref[:, 1])
    assert err <= TOL[precision], f"K2+Kf max relative error {err:.3e}"


@pytest.mark.parametrize(
    "overrides",
    [
        {"SYMMETRIZE_Z_Z2_INTEGRATION": False},
        {"NF": 0},
        {"ALPHA_S_CAP": 0.7},
    ],
)
def test_k2kf_and_k1_config_variants(overrides):
    config, r, N = _setup(rpoints=60, **overrides)
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    phys = oracle.physics(config)
    active = (np.arange(rn.size) > 0) & (Nn <= 0.99999)
    samples = 2048
    for precision in PRECISIONS:
        f32 = precision == _native.PRECISION_MIXED
        got = kernels.k2kf(r, N, config, samples=samples, precision=precision).cpu().numpy()
        lower, width = oracle.nlo_box(rn)
        ref = oracle.k2kf_sums(rn[active], _sobol_points(samples, 0, f32), lower, width, f32,
                               oracle.loglog_spline(rn, Nn, 1), phys)
        err = _rel_err(got[active, 0] + got[active, 1], ref[:, 0] + ref[:, 1])
        assert err <= TOL[precision], f"{overrides} K2+Kf {err:.3e}"
        k1 = kernels.k1(r, N, config, precision=precision).cpu().numpy()
        k1_ref = oracle.k1_fixed(rn[active], oracle.loglog_spline(rn, Nn, 0), phys)
        err = _rel_err(k1[active], k1_ref)
        assert err <= TOL[precision], f"{overrides} K1 {err:.3e}"


@pytest.mark.parametrize("precision", PRECISIONS)
def test_rhs_matches_oracle_derivative(precision):
    config, r, N = _setup(rpoints=99, MCINTPOINTS=2048)
    dndy, k1, k2kf = rhs(N, r, config, seed=0, precision=precision)
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    f32 = precision == _native.PRECISION_MIXED
    ref = oracle.derivative(Nn, rn, oracle.physics(config), _sobol_points(2048, 0, f32), f32)
    active = ref.dNdy != 0
    assert _rel_err(k1.cpu().numpy()[active], ref.K1[active]) <= TOL[precision]
    assert _rel_err(k2kf.cpu().numpy()[active], (ref.K2 + ref.Kf)[active]) <= TOL[precision]
    assert _rel_err(dndy.cpu().numpy()[active], ref.dNdy[active]) <= TOL[precision]
    assert np.all(dndy.cpu().numpy()[~active] == 0.0)


@pytest.mark.parametrize("stepper", ["euler", "rk3", "rk4"])
def test_one_step_each_stepper(stepper):
    config, r, N = _setup(rpoints=49, MCINTPOINTS=1024, DE_SOLVER_STEP=0.2, STEPPER=stepper, PRECISION="fp64")
    table = solve_bk(MV(qs0sqr=0.2), 0.2, config, device=DEVICE, dtype=torch.float64, seed=0)
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    ys, ref = oracle.evolve(Nn, rn, oracle.physics(config), _sobol_points(1024, 0, False), False, 0.2, 0.2,
                            stepper=stepper)
    got = table.N.cpu().numpy()
    assert got.shape == ref.shape
    np.testing.assert_allclose(table.y.cpu().numpy(), ys, rtol=0, atol=1e-15)
    np.testing.assert_allclose(got[-1], ref[-1], rtol=1e-10, atol=1e-300)


@pytest.mark.parametrize("tolerances", [(1e-6, 1e-4), (1e-10, 1e-7)])
def test_adaptive_rk2_matches_oracle(tolerances):
    """The reference's adaptive RK2 (step doubling) over two output steps, FP64 build against
    the oracle's restatement: the default DE_SOLVER_ABSERR / RELERR, and tolerances tight
    enough that attempts are rejected and h shrinks."""
    abserr, relerr = tolerances
    config, r, N = _setup(rpoints=49, MCINTPOINTS=1024, DE_SOLVER_STEP=0.2, STEPPER="rk2_adaptive",
                          PRECISION="fp64", DE_SOLVER_ABSERR=abserr, DE_SOLVER_RELERR=relerr)
    table = solve_bk(MV(qs0sqr=0.2), 0.4, config, device=DEVICE, dtype=torch.float64, seed=0)
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    _, ref = oracle.evolve(Nn, rn, oracle.physics(config), _sobol_points(1024, 0, False), False, 0.2, 0.4,
                           stepper="rk2_adaptive", abserr=abserr, relerr=relerr)
    got = table.N.cpu().numpy()
    assert got.shape == ref.shape == (3, rn.size)
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-300)
    # bk_steps keeps h from one output step to the next, as the reference's generator does
    from nlo_bk_optimized_b200.bk.evolution import bk_steps
    from nlo_bk_optimized_b200.dipole.table import DipoleTable

    start = DipoleTable(r=r, y=torch.zeros(1, dtype=torch.float64, device=DEVICE), N=N.unsqueeze(0), x0=0.01)
    last = list(bk_steps(start, 0.4, config, seed=0))[-1]
    np.testing.assert_allclose(last.N.cpu().numpy(), ref, rtol=1e-10, atol=1e-300)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_short_evolution_matches_oracle(precision):
    config, r, N = _setup(rpoints=79, MCINTPOINTS=2048, DE_SOLVER_STEP=0.2, PRECISION=precision)
    table = solve_bk(MV(qs0sqr=0.2), 1.0, config, device=DEVICE, dtype=torch.float64, seed=0)
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    f32 = precision == "mixed"
    _, ref = oracle.evolve(Nn, rn, oracle.physics(config), _sobol_points(2048, 0, f32), f32, 0.2, 1.0)
    got = table.N.cpu().numpy()
    tol = 1e-4 if f32 else 1e-10
    err = float(np.max(np.abs(got[-1] - ref[-1]) / np.maximum(np.abs(ref[-1]), 1e-300)))
    assert err <= tol, f"N(Y=1) max relative error {err:.3e}"


@pytest.mark.parametrize("stepper, precision", [("euler", "fp64"), ("rk3", "mixed"), ("rk4", "mixed"), ("rk4", "fp64")])
def test_replayed_steps_equal_launched_steps(stepper, precision):
    """An evolution on more than 192 points launches its first step kernel by kernel and
    replays a CUDA graph of one step for the later ones; one-step calls (launched kernel by
    kernel every time) give the same rows bit for bit."""
    config, _, _ = _setup(rpoints=199, MCINTPOINTS=2048, DE_SOLVER_STEP=0.2, STEPPER=stepper, PRECISION=precision)
    whole = solve_bk(MV(qs0sqr=0.2), 1.0, config, device=DEVICE, dtype=torch.float64, seed=0)
    part = solve_bk(MV(qs0sqr=0.2), 0.2, config, device=DEVICE, dtype=torch.float64, seed=0)
    for y in (0.4, 0.6, 0.8, 1.0):
        part = evolve_table(part, y, config, seed=0)
    assert whole.N.shape == part.N.shape == (6, 200)
    assert torch.equal(whole.N, part.N)
    assert not torch.equal(whole.N[-1], whole.N[1])


def test_deterministic_and_seeded():
    config, r, N = _setup(rpoints=99)
    a = kernels.k2kf(r, N, config, samples=5000)
    b = kernels.k2kf(r, N, config, samples=5000)
    assert torch.equal(a, b)
    c = kernels.k2kf(r, N, config, samples=5000, seed=1)
    assert not torch.equal(a, c)


def test_public_api_shapes():
    config = BKConfig(RPOINTS=49, MCINTPOINTS=1024, DE_SOLVER_STEP=0.2)
    table = solve_bk(MV(qs0sqr=0.2), 0.4, config, device=DEVICE, dtype=torch.float32, seed=3)
    assert table.N.shape == (3, 50) and table.N.dtype == torch.float32 and table.N.is_cuda
    assert table.y.tolist() == pytest.approx([0.0, 0.2, 0.4])
    assert bool(((table.N >= 0) & (table.N <= 1)).all())
    longer = evolve_table(table, 0.6, config, seed=3)
    assert longer.N.shape == (4, 50)
    torch.testing.assert_close(longer.N[:3], table.N)
    d = compute_dndy(MV(qs0sqr=0.2), config, device=DEVICE, seed=3)
    assert d.r.numel() == d.K1.numel() == d.K2_Kf.numel() == d.N.numel()


def test_nonfinite_initial_condition_raises():
    config = BKConfig(RPOINTS=29, MCINTPOINTS=256, DE_SOLVER_STEP=0.2)

    class Broken(MV):
        def dipole_amplitude(self, r):
            out = super().dipole_amplitude(r)
            out[5] = float("nan")
            return out

    with pytest.raises(FloatingPointError):
        solve_bk(Broken(qs0sqr=0.2), 0.2, config, device=DEVICE, dtype=torch.float64)
