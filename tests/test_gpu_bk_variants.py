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
