"""Pin the CPU oracle against the reference's own outputs (tests/golden, made by
tests/golden/make_golden.py from torch_nlo_clean/src/nlo_torch) and against
quad-precision evaluations of the reference's literal formulas."""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from golden_data import bk_reference


class _Config:
    NC = 3.0
    NF = 3
    LambdaQCD = 0.241
    C2 = 1.0
    MINR = 1e-6
    KSUB = 0.65
    SYMMETRIZE_Z_Z2_INTEGRATION = True
    FIXED_AS = 0.2
    ALPHA_S_CAP = 0.0


PHYS = oracle.physics(_Config())


@pytest.fixture(scope="module")
def g():
    return bk_reference()


@pytest.fixture(scope="module")
def splines(g):
    return oracle.loglog_spline(g["r"], g["N_mv"], 0), oracle.loglog_spline(g["r"], g["N_mv"], 1)


def test_grid_and_initial_condition(g):
    r = oracle.r_grid(1e-6, 1e2, 99)
    np.testing.assert_array_equal(r, g["r"])
    np.testing.assert_allclose(oracle.mv_amplitude(r, 0.2), g["N_mv"], rtol=1e-15, atol=0)


def test_log_n_spline_matches_reference(g, splines):
    nspl, _ = splines
    np.testing.assert_allclose(nspl.x, g["nspline_x"], rtol=0, atol=0)
    for field in "abcd":
        np.testing.assert_allclose(getattr(nspl, field), g[f"nspline_{field}"], rtol=1e-13, atol=1e-13)


def test_log_s_spline_matches_reference_where_well_conditioned(g, splines):
    # The oracle forms log S = log1p(-N); the reference log(1 - N).  They agree to
    # absolute rounding (~1e-16) in log S, which the spline solve spreads smoothly.
    _, sspl = splines
    for field in "abcd":
        np.testing.assert_allclose(getattr(sspl, field), g[f"sspline_{field}"], rtol=1e-10, atol=1e-11)


def test_coupling_matches_reference(g):
    values = np.array([oracle.alpha_s(float(r), PHYS) for r in g["alpha_r"]])
    np.testing.assert_allclose(values, g["alpha_s"], rtol=1e-14, atol=0)


def test_bessel_functions_match_torch_special(g):
    i1 = np.array([oracle.bessel_i1(float(x)) for x in g["bessel_x"]])
    np.testing.assert_allclose(i1, g["bessel_i1"], rtol=1e-13, atol=1e-300)
    # The oracle calls the C library's j1 (glibc), which agrees with scipy to 1e-15.
    # torch.special.bessel_j1 in float64, which the reference calls, is off by up to
    # ~7e-8 absolute on 3 < x < 20; that bounds K1 comparisons with the golden sums.
    from scipy.special import j1 as scipy_j1

    np.testing.assert_allclose(scipy_j1(g["bessel_x"]), g["bessel_j1"], rtol=0, atol=1e-7)


def test_sobol_points_bit_exact(g):
    state, shift = g["sobol_state"], g["sobol_shift"]
    f32 = oracle.sobol(state, shift, 0, 1024, as_f32=True)
    np.testing.assert_array_equal(f32.astype(np.float32), g["sobol_f32"])
    f64 = oracle.sobol(state, shift, 0, 1024, as_f32=False)
    np.testing.assert_array_equal(f64, g["sobol_f64"])
    # offsets continue the same sequence
    tail = oracle.sobol(state, shift, 500, 524, as_f32=False)
    np.testing.assert_array_equal(tail, g["sobol_f64"][500:])


def test_k2kf_integrand_matches_reference(g, splines):
    _, sspl = splines
    r = g["r"]
    for row, index in enumerate(g["k2kf_parent_index"]):
        if r[index] < 1e-3:
            # below ~1e-3 the reference's literal FP64 kernel carries relative rounding
            # noise ~eps (z/r)^2; the quad-precision tests below pin that regime
            continue
        ref = g["k2kf_value"][row]
        mine = np.array([sum(oracle.k2kf_integrand(float(r[index]), x, sspl, PHYS)) for x in g["k2kf_x"]])
        scale = np.abs(ref).max()
        # per-sample agreement relative to the integrand's scale, and on the sum
        assert np.max(np.abs(mine - ref)) <= 1e-8 * scale, index
        assert abs(mine.sum() - ref.sum()) <= 1e-10 * np.abs(ref).sum(), index


def test_k1_fixed_rule_matches_reference_sum(g, splines):
    nspl, _ = splines
    r = g["r"]
    mine = oracle.k1_fixed(r[g["k1_fixed_parent_index"]], nspl, PHYS)
    np.testing.assert_allclose(mine, g["k1_fixed"], rtol=1e-7, atol=0)


def test_k1_fixed_rule_close_to_reference_adaptive_integral(g, splines):
    nspl, _ = splines
    fixed = oracle.k1_fixed(g["r"][60:61], nspl, PHYS)[0]
    value, error = g["k1_adaptive_r60"]
    # the adaptive reference targets 1e-3 relative accuracy (BKConfig.INTACCURACY)
    assert abs(fixed - value) <= max(5 * error, 2e-3 * abs(value))


def test_k1_integrand_matches_reference_pointwise(g, splines):
    nspl, _ = splines
    r = g["r"]
    for row, index in enumerate(g["k1_parent_index"][:3]):
        ref = g["k1_value"][row]
        mine = np.array([oracle.k1_integrand(float(r[index]), float(z), float(t), nspl, PHYS)
                         for z, t in zip(g["k1_z"], g["k1_theta"])])
        scale = np.abs(ref).max()
        assert np.max(np.abs(mine - ref)) <= 1e-8 * scale, index


def test_lo_kernel_matches_reference(g):
    r = g["r"]
    for row, index in enumerate(g["k1_parent_index"]):
        mine = np.array([oracle.lo_kernel(float(r[index]), float(z), float(t), PHYS)
                         for z, t in zip(g["k1_z"], g["k1_theta"])])
        np.testing.assert_allclose(mine, g["kernel_lo"][row], rtol=2e-7, atol=0)


@pytest.mark.parametrize("parent", [1e-6, 1e-3, 1.0, 50.0])
def test_stable_nlo_kernels_equal_quad_literal(parent):
    """The cancellation-free K2/Kf forms equal the reference formulas evaluated in
    quad precision (where quad itself is well conditioned, t > 1e-8)."""

    rng = np.random.default_rng(7)
    lo, hi = math.log(0.5e-6), math.log(200.0)
    worst = 0.0
    for _ in range(400):
        x = np.array([rng.uniform(lo, hi), rng.uniform(lo, hi), rng.uniform(0, 2 * math.pi),
                      rng.uniform(0, 2 * math.pi)])
        stable = oracle.nlo_kernels(parent, *x)
        quad = oracle.nlo_kernels_literal_quad(parent, *x)
        worst = max(worst, float(np.max(np.abs(stable - quad) / np.abs(quad))))
    assert worst < (1e-6 if parent < 1e-4 else 1e-9)


@pytest.mark.parametrize("parent", [1e-6, 1e-3, 1.0])
def test_stable_lo_kernel_equals_quad_literal(parent):
    rng = np.random.default_rng(8)
    worst = 0.0
    for _ in range(300):
        z = math.exp(rng.uniform(math.log(1e-6), math.log(100.0)))
        t = rng.uniform(0, math.pi)
        worst = max(worst, abs(oracle.lo_kernel(parent, z, t, PHYS) / oracle.lo_kernel_literal_quad(parent, z, t, PHYS) - 1))
    assert worst < 1e-12


@pytest.mark.parametrize("qs", [0.2, 20.0])
def test_stable_dipoles_equal_quad_literal(qs):
    r = oracle.r_grid(1e-7, 1e2, 399)
    N = oracle.mv_amplitude(r, qs)
    nspl = oracle.loglog_spline(r, N, 0)
    sspl = oracle.loglog_spline(r, N, 1)
    lower, width = oracle.nlo_box(r)
    rng = np.random.default_rng(3)
    for index in (1, 50, 150, 250, 330, 380):
        for _ in range(150):
            z = math.exp(rng.uniform(math.log(r[0]), math.log(r[-1])))
            t = rng.uniform(0, math.pi)
            stable, quad = oracle.k1_dipole(nspl, r[index], z, t)
            assert abs(stable - quad) <= 4e-15 * max(abs(quad), 5e-2) + 1e-30
            x = lower + width * rng.uniform(0, 1, 4)
            s2, q2 = oracle.k2_dipoles(sspl, r[index], x)
            assert np.all(np.abs(s2 - q2) <= 1e-14 + 1e-9 * np.abs(q2))


def test_rk3_known_answer(monkeypatch):
    """bk/evolution.py:190-236 with a constant derivative 2: one step of 0.2 adds 0.4
    (the reference's own test, T/tests/test_bk_production.py:22-49)."""

    class _D:
        def __init__(self, n):
            self.dNdy = np.full(n, 2.0)

    monkeypatch.setattr(oracle, "derivative", lambda N, *a, **k: _D(N.size))
    N0 = np.array([0.3, 0.4])
    for stepper in ("rk3", "rk4", "euler"):
        ys, table = oracle.evolve(N0, np.array([0.1, 0.2]), PHYS, np.zeros((1, 4)), False, 0.2, 0.2,
                                  stepper=stepper, force_positive=False)
        np.testing.assert_allclose(table[-1], N0 + 0.4, rtol=1e-15)
        assert ys.tolist() == pytest.approx([0.0, 0.2])
