"""Pin the DIS oracle (oracle/dis.py) to values produced by the reference itself.

The fixture ``tests/golden/dis_reference.npz`` was written by
``tests/golden/make_golden_dis.py`` with the reference package on the CPU in float64.
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import dis as od

GOLDEN = np.load(Path(__file__).parent / "golden" / "dis_reference.npz")


def kin_of(name: str) -> tuple[od.Kinematics, float]:
    k = GOLDEN[f"{name}/kin"]
    kin = od.Kinematics(Q2=k[0], xbj=k[1], mf=k[2], transverse=bool(k[4]), maxr=k[5], finite_nc=bool(k[6]),
                        parent_coupling=bool(k[7]), smooth_coupling=bool(k[8]), c2_alpha=k[9],
                        active_flavors=int(k[10]), max_alpha=k[11])
    return kin, float(k[3])


def table_dipole() -> od.TableDipole:
    return od.TableDipole(GOLDEN["table_r"], GOLDEN["table_y"], GOLDEN["table_N"])


def gbw_dipole() -> od.GBWDipole:
    q, lam, g, x0 = GOLDEN["gbw_params"]
    return od.GBWDipole(qs0sqr=q, lam=lam, gamma=g, x0=x0)


def dipole_for(name: str):
    return table_dipole() if name.endswith("bk") or "_bk_" in name else gbw_dipole()


def rel(a, b, floor):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))


CASES = [str(c) for c in GOLDEN["cases"]]


def test_special_functions():
    assert rel(od.li2(GOLDEN["li2_x"]), GOLDEN["li2"], 1e-300) < 1e-13
    assert rel(od.k0(GOLDEN["bessel_x"]), GOLDEN["k0"], 1e-300) < 1e-13
    assert rel(od.k1(GOLDEN["bessel_x"]), GOLDEN["k1"], 1e-300) < 1e-13


def test_couplings():
    r = GOLDEN["alpha_r"]
    assert rel(od.alpha_freeze(r, 3, 1.0, 0.7), GOLDEN["alpha_freeze"], 0) < 1e-14
    assert rel(od.alpha_smooth(r, 4, 2.0), GOLDEN["alpha_smooth"], 0) < 1e-14


def test_amplitudes():
    r, Y = GOLDEN["amp_r"], GOLDEN["amp_Y"]
    assert rel(gbw_dipole()(r, Y), GOLDEN["gbw"], 1e-300) < 1e-13
    tab = table_dipole()
    assert rel(tab(r, Y), GOLDEN["amp_local"], 1e-12) < 1e-11
    tab.initialize(float(GOLDEN["amp_init_Y"][0]))
    assert tab.maxr_interpolate == pytest.approx(float(GOLDEN["amp_init_maxr"][0]), rel=1e-12)
    assert rel(tab(r, np.full_like(r, GOLDEN["amp_init_Y"][0])), GOLDEN["amp_init"], 1e-12) < 1e-11


def bilinear_dipole() -> od.TableDipole:
    return od.TableDipole(GOLDEN["table_r"], GOLDEN["table_y"], GOLDEN["table_N"], interpolation="linear_linear")


def test_bilinear_amplitudes():
    r, Y = GOLDEN["bilin_r"], GOLDEN["bilin_Y"]
    tab = bilinear_dipole()
    assert rel(tab(r, Y), GOLDEN["bilin_amp"], 1e-12) < 1e-12
    assert tab(np.array([GOLDEN["table_r"][-1]]), np.array([3.0]))[0] == 1.0  # the last knot
    tab.initialize(4.7)
    assert tab.maxr_interpolate == pytest.approx(float(GOLDEN["bilin_init_maxr"][0]), rel=1e-12)
    assert rel(tab(r, np.full_like(r, 4.7)), GOLDEN["bilin_init"], 1e-12) < 1e-11


def test_bilinear_dipole_term_and_lo():
    kin, _ = kin_of("light_T_bk")  # Q2 = 10, x = 1e-3, light quark, default couplings
    x = GOLDEN["bilin_dip1_x"]
    ref = GOLDEN["bilin_dip1"]
    got = od.dip_integrand(x, kin, 1, bilinear_dipole())
    assert rel(got, ref, 1e-9 * np.max(np.abs(ref))) < 1e-9
    Q2, xbj = 7.5, 2e-4
    quarks = [(0.14, 2 / 3), (1.4, 4 / 9)]
    dip = bilinear_dipole()
    dip.initialize(max(math.log(dip.X0() / xbj), 0.0))
    for transverse, want in zip((True, False), GOLDEN["bilin_lo_sf"]):
        sigma = od.LO_FACTOR * od.gauss_legendre_tensor(
            lambda u: od.lo_integrand(u, Q2, xbj, quarks, transverse, dip), 2, 24)
        assert sigma * od.structure_function_factor(Q2) == pytest.approx(want, rel=1e-12)


@pytest.mark.parametrize("name", CASES)
def test_lo_integrand(name):
    kin, e2 = kin_of(name)
    dip = dipole_for(name)
    if isinstance(dip, od.TableDipole):
        dip.initialize(max(math.log(dip.X0() / kin.xbj), 0.0))
    x = GOLDEN[f"{name}/lo_x"]
    got = od.lo_integrand(x, kin.Q2, kin.xbj, [(kin.mf, e2)], kin.transverse, dip, kin.maxr)
    ref = GOLDEN[f"{name}/lo"]
    assert rel(got, ref, 1e-12 * np.max(np.abs(ref))) < 1e-11
    sigma = od.LO_FACTOR * od.gauss_legendre_tensor(
        lambda u: od.lo_integrand(u, kin.Q2, kin.xbj, [(kin.mf, e2)], kin.transverse, dip, kin.maxr), 2, 24)
    assert sigma == pytest.approx(float(GOLDEN[f"{name}/sigma_lo"][0]), rel=1e-12)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("order", [0, 1, 2])
def test_dipole_terms(name, order):
    kin, _ = kin_of(name)
    x = GOLDEN[f"{name}/dip{order}_x"]
    got = od.dip_integrand(x, kin, order, dipole_for(name))
    ref = GOLDEN[f"{name}/dip{order}"]
    assert np.all(np.isfinite(ref))
    assert rel(got, ref, 1e-9 * np.max(np.abs(ref))) < 1e-9


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("term", ["I1", "I2", "I3"])
def test_qg_terms(name, term):
    kin, _ = kin_of(name)
    x = GOLDEN[f"{name}/qg_{term}_x"]
    got = od.qg_integrand(x, kin, term, dipole_for(name))
    ref = GOLDEN[f"{name}/qg_{term}"]
    assert rel(got, ref, 1e-9 * np.max(np.abs(ref))) < 1e-9


def test_nested_rule_matches_unnested_integral():
    """The nested I2/I3 forms equal the un-nested integrands integrated over the extra
    variables with the same inner rule (the reference's nesting, dis/observables.py:253-331)."""
    name = CASES[0]
    kin, _ = kin_of(name)
    dip = dipole_for(name)
    x5 = np.random.default_rng(3).uniform(0.05, 0.95, (6, 5))
    ys, ws = od.nested_rule(48)
    i2 = od.qg_integrand(x5, kin, "I2n", dip)
    i3 = od.qg_integrand(x5, kin, "I3n", dip)
    acc2 = np.zeros(6)
    acc3 = np.zeros(6)
    for y1, w1 in zip(ys, ws):
        acc2 += w1 * od.qg_integrand(np.column_stack([x5, np.full(6, y1)]), kin, "I2", dip)
        for y2, w2 in zip(ys, ws):
            acc3 += w1 * w2 * od.qg_integrand(np.column_stack([x5, np.full(6, y1), np.full(6, y2)]), kin, "I3", dip)
    assert rel(i2, acc2, 1e-12 * np.max(np.abs(acc2))) < 1e-10
    assert rel(i3, acc3, 1e-12 * np.max(np.abs(acc3))) < 1e-10


def test_vegas_driver_matches_reference_run():
    """The oracle's Vegas driver, fed the reference's own random draws
    (torch.randint bins then torch.rand fractions, numerics/integration.py:249-260),
    reproduces the reference run recorded in the fixture."""
    value, error, n_eval, converged, seed, samples, iters, bins = GOLDEN["vegas_pin"]
    kin = od.Kinematics(Q2=10.0, xbj=1e-3, mf=0.14, transverse=True, active_flavors=3)
    dip = gbw_dipole()
    gen = torch.Generator()
    gen.manual_seed(int(seed))

    def sampler(it, n):
        bi = torch.randint(int(bins), (n, 3), generator=gen)
        fr = torch.rand((n, 3), dtype=torch.float64, generator=gen)
        return bi.numpy(), fr.numpy()

    got = od.vegas(lambda x: od.dip_integrand(x, kin, 1, dip), 3, sampler, samples=int(samples),
                   max_iterations=int(iters), min_iterations=int(iters), bins=int(bins), epsrel=1e-9)
    assert got[0] == pytest.approx(value, rel=1e-11)
    assert got[1] == pytest.approx(error, rel=1e-9)
    assert got[2] == n_eval
    assert np.max(np.abs(got[4] - GOLDEN["vegas_pin_edges"])) < 1e-12


@pytest.mark.parametrize("kind", ["gbw", "bk"])
def test_lo_structure_functions(kind):
    FTv, FLv, F2v = GOLDEN[f"lo_sf_{kind}"]
    Q2, xbj = 7.5, 2e-4
    quarks = [(0.14, 2 / 3), (1.4, 4 / 9)]
    dip = gbw_dipole() if kind == "gbw" else table_dipole()
    if kind == "bk":
        dip.initialize(max(math.log(dip.X0() / xbj), 0.0))
    out = []
    for transverse in (True, False):
        sigma = od.LO_FACTOR * od.gauss_legendre_tensor(
            lambda u: od.lo_integrand(u, Q2, xbj, quarks, transverse, dip), 2, 24)
        out.append(sigma * od.structure_function_factor(Q2))
    assert out[0] == pytest.approx(FTv, rel=1e-12)
    assert out[1] == pytest.approx(FLv, rel=1e-12)
    assert out[0] + out[1] == pytest.approx(F2v, rel=1e-12)


def test_fixed_sobol_sampling_pieces():
    """map_importance_grid, paired_endpoint_inputs and the grid re-binning against the
    reference's own functions."""
    src, inv, bi = od.map_importance_grid(GOLDEN["fs_points"], GOLDEN["fs_edges"])
    assert np.array_equal(bi, GOLDEN["fs_bins"])
    assert rel(src, GOLDEN["fs_source"], 1e-300) < 1e-14
    assert rel(inv, GOLDEN["fs_inv"], 1e-300) < 1e-13
    for fold in (False, True):
        tag = "fold" if fold else "nofold"
        f, fw, s, sw = od.paired_endpoint_inputs(GOLDEN["fs_source"], 5.0, fold)
        assert rel(f, GOLDEN[f"fs_first_{tag}"], 1e-300) < 1e-13
        assert rel(fw, GOLDEN[f"fs_fw_{tag}"], 1e-300) < 1e-13
        assert rel(s, GOLDEN[f"fs_second_{tag}"], 1e-12) < 1e-12
        assert rel(sw, GOLDEN[f"fs_sw_{tag}"], 1e-300) < 1e-12
    new = od.adapt_edges(GOLDEN["fs_edges"], GOLDEN["adapt_hist"], GOLDEN["adapt_count"])
    assert np.max(np.abs(new - GOLDEN["adapt_edges"])) < 1e-15


def test_fixed_sobol_replicate_statistics_known_answer():
    """The correlated-replicate total of T/tests/test_dis_production.py:153-192: replicate
    totals (0.7, 0.7, 0.65) give their mean and std/sqrt(3)."""
    mean, err = od.replicate_result([0.7, 0.7, 0.65])
    assert mean == pytest.approx(np.mean([0.7, 0.7, 0.65]), rel=1e-15)
    assert err == pytest.approx(np.std([0.7, 0.7, 0.65], ddof=1) / math.sqrt(3), rel=1e-15)
