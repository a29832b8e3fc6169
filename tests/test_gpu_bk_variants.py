"""Parity of the device K1, K2+Kf, right-hand side and evolution with the oracle for the
non-production BKConfig choices: every Order, RC_LO and RESUM_RC, RC_NLO = PARENT_NLO and
NF = 5 (the oracle is pinned on the reference's own values for the same choices in
test_oracle_variants.py).  Tolerances as for the production choice: 1e-10 relative for
the all-FP64 build, 1e-4 for the mixed build."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from golden_data import bk_variants, variant_config
from nlo_bk_optimized_b200 import MV, _native, kernels, solve_bk
from nlo_bk_optimized_b200.bk.evolution import _r_grid, rhs

pytestmark = pytest.mark.gpu

TOL = {_native.PRECISION_MIXED: 1e-4, _native.PRECISION_FP64: 1e-10}
PRECISIONS = [_native.PRECISION_MIXED, _native.PRECISION_FP64]
NAMES = [str(n) for n in bk_variants()["names"]]
# the choices that reach K2 + Kf
K2_NAMES = ["rc_nlo_parent", "nf5", "rc_fixed", "nf5_fac_dlog"]


def _rel_err(gpu, ref, floor=1e-3):
    scale = np.maximum(np.abs(ref), floor * np.max(np.abs(ref)) + 1e-300)
    return float(np.max(np.abs(gpu - ref) / scale))


def _grid(config):
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    N = MV(qs0sqr=0.2).dipole_amplitude(r)
    rn, Nn = r.cpu().numpy(), N.cpu().numpy()
    active = (np.arange(rn.size) > 0) & (Nn <= 0.99999)
    return r, N, rn, Nn, active


def _sobol(n, f32):
    state, shift = oracle.sobol_state(4, 0)
    return oracle.sobol(state, shift, 0, n, as_f32=f32)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("precision", PRECISIONS)
def test_k1_variant_matches_oracle(name, precision):
    config = variant_config(name)
    r, N, rn, Nn, active = _grid(config)
    got = kernels.k1(r, N, config, precision=precision).cpu().numpy()
    ref = oracle.k1_fixed(rn[active], oracle.loglog_spline(rn, Nn, 0), oracle.physics(config))
    assert np.all(got[~active] == 0.0)
    err = _rel_err(got[active], ref)
    assert err <= TOL[precision], f"{name}: K1 max relative error {err:.3e}"


@pytest.mark.parametrize("name", K2_NAMES)
@pytest.mark.parametrize("precision", PRECISIONS)
def test_k2kf_variant_matches_oracle(name, precision):
    config = variant_config(name)
    r, N, rn, Nn, active = _grid(config)
    samples = 2048
    f32 = precision == _native.PRECISION_MIXED
    got = kernels.k2kf(r, N, config, samples=samples, precision=precision).cpu().numpy()
    lower, width = oracle.nlo_box(rn)
    ref = oracle.k2kf_sums(rn[active], _sobol(samples, f32), lower, width, f32, oracle.loglog_spline(rn, Nn, 1),
                           oracle.physics(config))
    for label, a, b in (("K2", got[active, 0], ref[:, 0]), ("Kf", got[active, 1], ref[:, 1]),
                        ("K2+Kf", got[active, 0] + got[active, 1], ref[:, 0] + ref[:, 1])):
        err = _rel_err(a, b)
        assert err <= TOL[precision], f"{name}: {label} max relative error {err:.3e}"


@pytest.mark.parametrize("name", ["order_lo", "order_lo_dlog", "order_lo_dlog_slog", "order_nlo", "nf5_fac_dlog"])
@pytest.mark.parametrize("precision", PRECISIONS)
def test_rhs_variant_matches_oracle(name, precision):
    """Orders without NLO kernels take no K2 + Kf; the others add it (bk/evolution.py:391, 473)."""
    from dataclasses import replace

    config = replace(variant_config(name), MCINTPOINTS=1024)
    r, N, rn, Nn, active = _grid(config)
    dndy, k1, k2kf = rhs(N, r, config, seed=0, precision=precision)
    f32 = precision == _native.PRECISION_MIXED
    ref = oracle.derivative(Nn, rn, oracle.physics(config), _sobol(1024, f32), f32)
    k2kf = k2kf.cpu().numpy()
    if config.Order.has_nlo_kernels:
        assert _rel_err(k2kf[active], (ref.K2 + ref.Kf)[active]) <= TOL[precision]
    else:
        assert np.all(k2kf == 0.0) and np.all(ref.K2 == 0.0)
    assert _rel_err(k1.cpu().numpy()[active], ref.K1[active]) <= TOL[precision]
    assert _rel_err(dndy.cpu().numpy()[active], ref.dNdy[active]) <= TOL[precision]


@pytest.mark.parametrize("name", ["order_lo", "nf5_fac_dlog", "smallest_beuf_parent"])
def test_short_variant_evolution_matches_oracle(name):
    from dataclasses import replace

    config = replace(variant_config(name), RPOINTS=59, MCINTPOINTS=1024, DE_SOLVER_STEP=0.2, PRECISION="fp64")
    r, N, rn, Nn, _ = _grid(config)
    table = solve_bk(MV(qs0sqr=0.2), 0.6, config, device="cuda", dtype=torch.float64, seed=0)
    _, ref = oracle.evolve(Nn, rn, oracle.physics(config), _sobol(1024, False), False, 0.2, 0.6)
    got = table.N.cpu().numpy()
    assert got.shape == ref.shape
    err = float(np.max(np.abs(got[-1] - ref[-1]) / np.maximum(np.abs(ref[-1]), 1e-300)))
    assert err <= 1e-10, f"{name}: N(Y=0.6) max relative error {err:.3e}"


# ----------------------------------------------------------------------------- kinematical constraint
def _kc_history(config):
    g = bk_variants()
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    assert np.allclose(r.cpu().numpy(), g["r"], rtol=1e-15)
    return r, g["kc_history_y"], g["kc_history_N"]


@pytest.mark.parametrize("name", [str(n) for n in bk_variants()["kc_names"]])
@pytest.mark.parametrize("precision", PRECISIONS)
def test_kinematical_constraint_rhs_matches_oracle(name, precision):
    from dataclasses import replace

    config = replace(variant_config(name), MCINTPOINTS=1024)
    r, hy, hN = _kc_history(config)
    rn = r.cpu().numpy()
    N = torch.tensor(hN[-1], device="cuda")
    history = (torch.tensor(hy, device="cuda"), torch.tensor(hN, device="cuda"))
    dndy, k1, k2kf = rhs(N, r, config, seed=0, precision=precision, history=history)
    f32 = precision == _native.PRECISION_MIXED
    ref = oracle.derivative(hN[-1], rn, oracle.physics(config), _sobol(1024, f32), f32, history=(hy, hN))
    active = ref.dNdy != 0
    assert _rel_err(k1.cpu().numpy()[active], ref.K1[active]) <= TOL[precision]
    # dN/dY = K1 + (K2+Kf) cancels at some parents: measure its error against the parts
    parts = np.abs(ref.K1) + np.abs(ref.K2 + ref.Kf)
    err = np.abs(dndy.cpu().numpy() - ref.dNdy)[active] / parts[active]
    assert float(err.max()) <= TOL[precision]
    with pytest.raises(ValueError):
        rhs(N, r, config, seed=0, precision=precision)  # the constraint needs the history


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_kinematical_constraint_evolution_matches_oracle(precision):
    from dataclasses import replace

    config = replace(variant_config("kc"), RPOINTS=59, MCINTPOINTS=1024, DE_SOLVER_STEP=0.2, PRECISION=precision)
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    rn = r.cpu().numpy()
    N0 = MV(qs0sqr=0.2).dipole_amplitude(r).cpu().numpy()
    table = solve_bk(MV(qs0sqr=0.2), 0.8, config, device="cuda", dtype=torch.float64, seed=0)
    f32 = precision == "mixed"
    ys, ref = oracle.evolve(N0, rn, oracle.physics(config), _sobol(1024, f32), f32, 0.2, 0.8, stepper="euler",
                            kinematical_constraint=True)
    got = table.N.cpu().numpy()
    assert got.shape == ref.shape
    tol = 1e-4 if f32 else 1e-10
    err = float(np.max(np.abs(got[-1] - ref[-1]) / np.maximum(np.abs(ref[-1]), 1e-300)))
    assert err <= tol, f"N(Y=0.8) max relative error {err:.3e}"
    # the constraint changes the evolution
    _, plain = oracle.evolve(N0, rn, oracle.physics(replace(config, KINEMATICAL_CONSTRAINT=False)),
                             _sobol(1024, f32), f32, 0.2, 0.8, stepper="euler")
    assert np.max(np.abs(plain[-1] - ref[-1]) / np.maximum(np.abs(ref[-1]), 1e-300)) > 1e-3


def test_kinematical_constraint_continuation_equals_one_run():
    """evolve_table carries the stored rows as the constraint's history."""
    from dataclasses import replace

    from nlo_bk_optimized_b200.bk.evolution import evolve_table

    config = replace(variant_config("kc"), RPOINTS=49, MCINTPOINTS=512, DE_SOLVER_STEP=0.2, PRECISION="fp64")
    whole = solve_bk(MV(qs0sqr=0.2), 0.8, config, device="cuda", dtype=torch.float64, seed=0)
    part = solve_bk(MV(qs0sqr=0.2), 0.4, config, device="cuda", dtype=torch.float64, seed=0)
    resumed = evolve_table(part, 0.8, config, seed=0)
    np.testing.assert_array_equal(resumed.y.cpu().numpy(), whole.y.cpu().numpy())
    np.testing.assert_array_equal(resumed.N.cpu().numpy(), whole.N.cpu().numpy())


def test_kinematical_constraint_dndy_at_the_initial_rapidity():
    """At y = 0 the shifted rapidity is negative wherever min(X, Y) > r: only the rest of
    the K1 integral remains (bk/evolution.py:76-79)."""
    from dataclasses import replace

    from nlo_bk_optimized_b200 import compute_dndy

    config = replace(variant_config("kc"), MCINTPOINTS=512)
    res = compute_dndy(MV(qs0sqr=0.2), config, device="cuda", dtype=torch.float64, seed=0)
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    rn = r.cpu().numpy()
    N0 = MV(qs0sqr=0.2).dipole_amplitude(r).cpu().numpy()
    active = (np.arange(rn.size) > 0) & (N0 <= 0.99999)
    ref = oracle.k1_fixed(rn[active], oracle.loglog_spline(rn, N0, 0), oracle.physics(config),
                          history=(np.zeros(1), N0[None]), r_grid=rn)
    assert _rel_err(res.K1.cpu().numpy(), ref) <= 1e-10
