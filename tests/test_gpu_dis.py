"""Parity of the device DIS path with the reference (golden vectors) and the oracle.

FP64 build: pointwise 1e-10 relative (floor 1e-10 of the largest value of the sample set),
Vegas value/error/grid 1e-10 against the oracle's Vegas on the same Sobol points.
Mixed build (FP32 integrands): sums over the sample sets within 1e-4 relative of FP64.
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import dis as od

pytestmark = pytest.mark.gpu

GOLDEN = np.load(Path(__file__).parent / "golden" / "dis_reference.npz")
CASES = [str(c) for c in GOLDEN["cases"]]
FP64_TOL = 1e-10
MIXED_SUM_TOL = 1e-4


@pytest.fixture(scope="module")
def lib():
    from nlo_bk_optimized_b200 import _native

    return _native.load()


def dev(a):
    return torch.as_tensor(np.asarray(a), dtype=torch.float64, device="cuda")


def table_obj():
    from nlo_bk_optimized_b200.dipole import BKDipole, DipoleTable

    t = DipoleTable(dev(GOLDEN["table_r"]), dev(GOLDEN["table_y"]), dev(GOLDEN["table_N"]), 1.0)
    return BKDipole(t)


def gbw_obj():
    from nlo_bk_optimized_b200.dipole import GBW

    q, lam, g, x0 = GOLDEN["gbw_params"]
    return GBW(Qs0sqr=float(q), lambda_=float(lam), gamma=float(g), x0=float(x0))


def config_of(name):
    from nlo_bk_optimized_b200.dis import (
        DISConfig,
        NcScheme,
        Quark,
        QuarkType,
        RunningCouplingIRScheme,
        RunningCouplingScheme,
    )

    k = GOLDEN[f"{name}/kin"]
    quark = Quark(QuarkType.C if k[2] > 1 else QuarkType.LIGHT, float(k[2]))
    config = DISConfig(
        quarks=(quark,), maxr=float(k[5]),
        nc_scheme=NcScheme.FiniteNC if k[6] else NcScheme.LargeNC,
        rc_scheme=RunningCouplingScheme.PARENT if k[7] else RunningCouplingScheme.SMALLEST,
        rc_ir_scheme=RunningCouplingIRScheme.SMOOTH if k[8] else RunningCouplingIRScheme.FREEZE,
        C2_alpha=float(k[9]), max_alpha_s_freeze=float(k[11]))
    return config, quark, float(k[0]), float(k[1]), bool(k[4])


def oracle_kin(name):
    k = GOLDEN[f"{name}/kin"]
    return od.Kinematics(Q2=k[0], xbj=k[1], mf=k[2], transverse=bool(k[4]), maxr=k[5], finite_nc=bool(k[6]),
                         parent_coupling=bool(k[7]), smooth_coupling=bool(k[8]), c2_alpha=k[9],
                         active_flavors=int(k[10]), max_alpha=k[11])


def oracle_dipole(name):
    if name.endswith("bk") or "_bk_" in name:
        return od.TableDipole(GOLDEN["table_r"], GOLDEN["table_y"], GOLDEN["table_N"])
    q, lam, g, x0 = GOLDEN["gbw_params"]
    return od.GBWDipole(qs0sqr=q, lam=lam, gamma=g, x0=x0)


def device_dipole(name):
    return table_obj() if name.endswith("bk") or "_bk_" in name else gbw_obj()


def rel_err(got, ref):
    got = np.asarray(got)
    ref = np.asarray(ref)
    floor = FP64_TOL * max(np.max(np.abs(ref)), 1e-300)
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), floor)))


def pol_of(transverse):
    from nlo_bk_optimized_b200.dis import Polarization

    return Polarization.T if transverse else Polarization.L


def evaluate(term, x, name, precision):
    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.dis.observables import _integrand, kinematics

    config, quark, Q2, xbj, transverse = config_of(name)
    kin = kinematics(Q2, xbj, pol_of(transverse), config, None if term == "LO" else quark)
    dipole = device_dipole(name)
    if term == "LO":
        dipole_init = dipole
        if hasattr(dipole_init, "initialize_interpolation"):
            dipole_init.initialize_interpolation(max(math.log(dipole.X0() / xbj), 0.0))
    return _integrand(_native.DIS_TERMS[term], dev(x), kin, dipole, config, precision=precision).cpu().numpy()


# ----------------------------------------------------------------------------- amplitudes


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_amplitudes(dtype):
    r, Y = dev(GOLDEN["amp_r"]), dev(GOLDEN["amp_Y"])
    tol = FP64_TOL if dtype == torch.float64 else 2e-5
    gbw = gbw_obj().dipole_amplitude(r.to(dtype), Y.to(dtype)).double().cpu().numpy()
    # 1 - exp(-a) in the reference loses ~1e-16 absolute for small a: allow that absolute slack
    slack = 4e-16 if dtype == torch.float64 else 1e-9
    assert np.all(np.abs(gbw - GOLDEN["gbw"]) <= tol * np.abs(GOLDEN["gbw"]) + slack)
    tab = table_obj()
    local = tab.dipole_amplitude(r, Y).cpu().numpy()
    assert rel_err(local, GOLDEN["amp_local"]) < 1e-12
    tab.initialize_interpolation(float(GOLDEN["amp_init_Y"][0]))
    assert tab.maxr_interpolate == pytest.approx(float(GOLDEN["amp_init_maxr"][0]), rel=1e-12)
    init = tab.dipole_amplitude(r, torch.full_like(r, float(GOLDEN["amp_init_Y"][0]))).cpu().numpy()
    assert rel_err(init, GOLDEN["amp_init"]) < 1e-12


@pytest.mark.parametrize("interpolation", ["spline_linear", "linear_linear"])
def test_table_irregular_grids(interpolation):
    """Tables whose r knots sit up to 0.9 % off the logarithmic grid (BKDipole accepts 1 %)
    and whose rows are unevenly spaced in Y: the device finds the r interval and the two
    rows from a uniform-grid guess, corrected against the knots or replaced by a search;
    amplitudes on and between the knots, below and above the r range and on the rows
    equal the oracle's (dipole/amplitude.py:135-252)."""
    from nlo_bk_optimized_b200.dipole import AmplitudeInterpolation, BKDipole, DipoleTable

    rng = np.random.default_rng(11)
    r = np.geomspace(1e-6, 50.0, 80) * (1.0 + 0.009 * rng.uniform(-1.0, 1.0, 80))
    r[0], r[1] = 1e-6, 1e-6 * (50.0 / 1e-6) ** (1 / 79)  # the check measures from the first ratio
    y = np.array([0.0, 0.05, 0.1, 0.9, 1.0, 3.5, 3.6, 7.0, 12.0])
    N = 1.0 - np.exp(-np.outer(0.3 * np.exp(0.3 * y), r * r) / 4.0)
    rr = np.exp(rng.uniform(math.log(5e-7), math.log(60.0), 3000))
    YY = rng.uniform(0.0, 12.0, 3000)
    rr[: r.size] = r
    YY[: y.size] = y
    YY[y.size : 2 * y.size] = y[::-1]
    mode = AmplitudeInterpolation.LINEAR_LINEAR if interpolation == "linear_linear" else None
    kwargs = {"interpolation": mode} if mode is not None else {}
    tab = BKDipole(DipoleTable(dev(r), dev(y), dev(N), 1.0), **kwargs)
    got = tab.dipole_amplitude(dev(rr), dev(YY)).cpu().numpy()
    ref = od.TableDipole(r, y, N, 1.0, interpolation=interpolation)(rr, YY)
    assert rel_err(got, ref) < 1e-12


@pytest.mark.parametrize("mode", [0, 1])
def test_table_clustered_r_grid_c_abi(lib, mode):
    """The C ABI takes any increasing r grid (BKDipole, like the reference, insists on a
    logarithmic one): on knots clustered in three bands the log-grid guess misses the
    interval by up to 20 and the lookup falls back to its search; amplitudes still equal
    the oracle's table (dipole/amplitude.py:135-252)."""
    import ctypes

    from nlo_bk_optimized_b200 import _native

    r = np.concatenate([np.geomspace(1e-6, 1e-3, 12), np.geomspace(1.1e-3, 2.0, 60), np.geomspace(2.3, 50.0, 8)])
    y = np.array([0.0, 0.05, 0.1, 0.9, 1.0, 3.5, 3.6, 7.0, 12.0])
    N = 1.0 - np.exp(-np.outer(0.3 * np.exp(0.3 * y), r * r) / 4.0)
    rng = np.random.default_rng(5)
    rr = np.exp(rng.uniform(math.log(5e-7), math.log(60.0), 3000))
    YY = rng.uniform(0.0, 12.0, 3000)
    rr[: r.size] = r
    table = torch.empty(int(lib.nlo_dis_table_doubles(r.size, y.size)), dtype=torch.float64, device="cuda")
    stream = _native.stream_handle(torch.device("cuda", torch.cuda.current_device()))
    r_dev, y_dev, N_dev = dev(r), dev(y), dev(N)  # held until the prepare kernel has read them
    _native.check(lib.nlo_dis_table_prepare_interpolated(r_dev.data_ptr(), y_dev.data_ptr(), N_dev.data_ptr(),
                                                         r.size, y.size, 1.0, mode, table.data_ptr(), stream))
    d = _native.Dipole()
    d.kind = _native.DIPOLE_TABLE
    d.table = table.data_ptr()
    d.nr, d.ny = r.size, y.size
    rd, Yd = dev(rr), dev(YY)
    out = torch.empty_like(rd)
    _native.check(lib.nlo_dis_dipole_amplitude(ctypes.byref(d), rd.data_ptr(), Yd.data_ptr(), rd.numel(),
                                                _native.PRECISION_FP64, out.data_ptr(), stream))
    ref = od.TableDipole(r, y, N, 1.0, interpolation="linear_linear" if mode else "spline_linear")(rr, YY)
    assert rel_err(out.cpu().numpy(), ref) < 1e-12


def bilinear_obj():
    from nlo_bk_optimized_b200.dipole import AmplitudeInterpolation, BKDipole, DipoleTable

    t = DipoleTable(dev(GOLDEN["table_r"]), dev(GOLDEN["table_y"]), dev(GOLDEN["table_N"]), 1.0)
    return BKDipole(t, interpolation=AmplitudeInterpolation.LINEAR_LINEAR)


def test_bilinear_table_interpolation():
    """LINEAR_LINEAR tables (dipole/amplitude.py:188-212): amplitudes on the local and the
    initialised path, edges included, a dipole term and LO F_T, F_L against the reference."""
    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.dis import FL, FT, DISConfig, Quark, QuarkType
    from nlo_bk_optimized_b200.dis.observables import _integrand, kinematics

    r, Y = dev(GOLDEN["bilin_r"]), dev(GOLDEN["bilin_Y"])
    tab = bilinear_obj()
    assert rel_err(tab.dipole_amplitude(r, Y).cpu().numpy(), GOLDEN["bilin_amp"]) < 1e-12
    tab.initialize_interpolation(4.7)
    assert tab.maxr_interpolate == pytest.approx(float(GOLDEN["bilin_init_maxr"][0]), rel=1e-12)
    init = tab.dipole_amplitude(r, torch.full_like(r, 4.7)).cpu().numpy()
    assert rel_err(init, GOLDEN["bilin_init"]) < 1e-12

    config, quark, Q2, xbj, transverse = config_of("light_T_bk")
    kin = kinematics(Q2, xbj, pol_of(transverse), config, quark)
    x = dev(GOLDEN["bilin_dip1_x"])
    got = _integrand(_native.DIS_TERMS["DIP1"], x, kin, bilinear_obj(), config, precision=_native.PRECISION_FP64)
    assert rel_err(got.cpu().numpy(), GOLDEN["bilin_dip1"]) < 1e-9
    mixed = _integrand(_native.DIS_TERMS["DIP1"], x, kin, bilinear_obj(), config, precision=_native.PRECISION_MIXED)
    assert abs(float(mixed.sum() / got.sum()) - 1) < MIXED_SUM_TOL

    config = DISConfig(quarks=(Quark(QuarkType.LIGHT, 0.14), Quark(QuarkType.C, 1.4)), precision="fp64")
    Q2t = torch.tensor(7.5, dtype=torch.float64, device="cuda")
    xt = torch.tensor(2e-4, dtype=torch.float64, device="cuda")
    ref = GOLDEN["bilin_lo_sf"]
    assert float(FT(Q2t, xt, bilinear_obj(), config).value) == pytest.approx(ref[0], rel=1e-11)
    assert float(FL(Q2t, xt, bilinear_obj(), config).value) == pytest.approx(ref[1], rel=1e-11)


# ----------------------------------------------------------------------------- integrands vs golden


@pytest.mark.parametrize("name", CASES)
def test_lo_integrand(name):
    from nlo_bk_optimized_b200 import _native

    got = evaluate("LO", GOLDEN[f"{name}/lo_x"], name, _native.PRECISION_FP64)
    # the golden LO values carry the case's single quark with charge^2 of its type
    assert rel_err(got, GOLDEN[f"{name}/lo"]) < FP64_TOL
    mixed = evaluate("LO", GOLDEN[f"{name}/lo_x"], name, _native.PRECISION_MIXED)
    assert abs(mixed.sum() / got.sum() - 1) < MIXED_SUM_TOL


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("order", [0, 1, 2])
def test_dipole_terms(name, order):
    from nlo_bk_optimized_b200 import _native

    x = GOLDEN[f"{name}/dip{order}_x"]
    ref = GOLDEN[f"{name}/dip{order}"]
    got = evaluate(f"DIP{order}", x, name, _native.PRECISION_FP64)
    assert rel_err(got, ref) < 1e-9
    mixed = evaluate(f"DIP{order}", x, name, _native.PRECISION_MIXED)
    assert abs(mixed.sum() / got.sum() - 1) < MIXED_SUM_TOL


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("term", ["I1", "I2", "I3"])
def test_qg_terms(name, term):
    from nlo_bk_optimized_b200 import _native

    x = GOLDEN[f"{name}/qg_{term}_x"]
    ref = GOLDEN[f"{name}/qg_{term}"]
    got = evaluate(term, x, name, _native.PRECISION_FP64)
    assert rel_err(got, ref) < 1e-9
    mixed = evaluate(term, x, name, _native.PRECISION_MIXED)
    assert abs(mixed.sum() / got.sum() - 1) < MIXED_SUM_TOL


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("term", ["I2N", "I3N"])
def test_nested_terms_vs_oracle(name, term):
    from nlo_bk_optimized_b200 import _native

    x = np.random.default_rng(11).uniform(0, 1, (128, 5))
    ref = od.qg_integrand(x, oracle_kin(name), {"I2N": "I2n", "I3N": "I3n"}[term], oracle_dipole(name))
    got = evaluate(term, x, name, _native.PRECISION_FP64)
    assert rel_err(got, ref) < 1e-9
    mixed = evaluate(term, x, name, _native.PRECISION_MIXED)
    assert abs(mixed.sum() / got.sum() - 1) < MIXED_SUM_TOL


# ----------------------------------------------------------------------------- integrals


@pytest.mark.parametrize("name", CASES)
def test_sigma_lo_gauss_legendre(name):
    from nlo_bk_optimized_b200.dis import DISConfig, photon_proton_cross_section_LO_d2b

    config, quark, Q2, xbj, transverse = config_of(name)
    config = DISConfig(**{**{f: getattr(config, f) for f in config.__dataclass_fields__}, "precision": "fp64"})
    res = photon_proton_cross_section_LO_d2b(torch.tensor(Q2, dtype=torch.float64, device="cuda"),
                                             torch.tensor(xbj, dtype=torch.float64, device="cuda"),
                                             pol_of(transverse), device_dipole(name), config)
    assert float(res.value) == pytest.approx(float(GOLDEN[f"{name}/sigma_lo"][0]), rel=1e-11)
    assert float(res.error) == pytest.approx(float(GOLDEN[f"{name}/sigma_lo"][1]), rel=1e-6, abs=1e-14)


@pytest.mark.parametrize("kind", ["gbw", "bk"])
def test_lo_structure_functions(kind):
    from nlo_bk_optimized_b200.dis import F2, FL, FT, DISConfig, Quark, QuarkType

    config = DISConfig(quarks=(Quark(QuarkType.LIGHT, 0.14), Quark(QuarkType.C, 1.4)), precision="fp64")
    dip = gbw_obj() if kind == "gbw" else table_obj()
    Q2 = torch.tensor(7.5, dtype=torch.float64, device="cuda")
    xbj = torch.tensor(2e-4, dtype=torch.float64, device="cuda")
    ref = GOLDEN[f"lo_sf_{kind}"]
    assert float(FT(Q2, xbj, dip, config).value) == pytest.approx(ref[0], rel=1e-11)
    assert float(FL(Q2, xbj, dip, config).value) == pytest.approx(ref[1], rel=1e-11)
    assert float(F2(Q2, xbj, dip, config).value) == pytest.approx(ref[2], rel=1e-11)
    mixed = DISConfig(quarks=config.quarks)
    assert float(F2(Q2, xbj, dip, mixed).value) == pytest.approx(ref[2], rel=MIXED_SUM_TOL)


def sobol_points(dims, seed, n):
    return torch.quasirandom.SobolEngine(dims, scramble=True, seed=seed).draw(n, dtype=torch.float64).numpy()


@pytest.mark.parametrize("term,order,name", [("DIP1", 1, "light_T_bk"), ("DIP2", 2, "charm_L_gbw"),
                                             ("I1", None, "light_T_bk"), ("I3N", None, "light_L_bk")])
def test_vegas_matches_oracle(term, order, name):
    """Device Vegas (FP64) vs the oracle's Vegas driver on the same Sobol points."""
    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.dis.observables import kinematics
    from nlo_bk_optimized_b200.numerics.integration import VegasOptions, state_results, vegas_terms

    config, quark, Q2, xbj, transverse = config_of(name)
    dims = _native.DIS_DIMS[_native.DIS_TERMS[term]]
    n, iters, bins, seed = 2048 if term == "I3N" else 8192, 3, 50, 5
    opts = VegasOptions(samples_per_iteration=n, max_iterations=iters, min_iterations=iters, bins=bins,
                        epsrel=1e-12, inner_points=48)
    kin = kinematics(Q2, xbj, pol_of(transverse), config, quark)
    dip = device_dipole(name)
    state = vegas_terms(_native.DIS_TERMS[term], [kin], dip.native(), opts, [seed],
                        precision=_native.PRECISION_FP64, device=torch.device("cuda"))
    res = state_results(state, _native.DIS_TERMS[term], bins)
    pts = sobol_points(dims, seed, n * iters)
    okin, odip = oracle_kin(name), oracle_dipole(name)
    if order is not None:
        f = lambda u: od.dip_integrand(u, okin, order, odip)  # noqa: E731
    else:
        f = lambda u: od.qg_integrand(u, okin, term, odip)  # noqa: E731
    value, error, n_eval, converged, edges = od.vegas(
        f, dims, lambda it, m: od.sobol_sampler(pts[it * m:(it + 1) * m], bins), samples=n, max_iterations=iters,
        min_iterations=iters, bins=bins, epsrel=1e-12)
    assert float(res["value"][0]) == pytest.approx(value, rel=1e-10)
    assert float(res["error"][0]) == pytest.approx(error, rel=1e-8)
    assert int(res["n_eval"][0]) == n_eval
    assert np.max(np.abs(res["edges"][0].cpu().numpy() - edges)) < 1e-10
    # mixed precision: one iteration on the uniform grid against the FP64 value
    one = VegasOptions(samples_per_iteration=n, max_iterations=1, min_iterations=1, bins=bins, epsrel=1e-12)
    vals = []
    for precision in (_native.PRECISION_FP64, _native.PRECISION_MIXED):
        st = vegas_terms(_native.DIS_TERMS[term], [kin], dip.native(), one, [seed], precision=precision,
                         device=torch.device("cuda"))
        vals.append(float(state_results(st, _native.DIS_TERMS[term], bins)["value"][0]))
    assert vals[1] == pytest.approx(vals[0], rel=MIXED_SUM_TOL)


def test_batch_matches_single_points():
    """Every point of a batched structure-function run equals the same point run alone
    (the batch changes only the CTA split of each integral's sums)."""
    from nlo_bk_optimized_b200.dis import F2, DISConfig, DISOrder, Quark, QuarkType, structure_functions

    config = DISConfig(order=DISOrder.NLO, quarks=(Quark(QuarkType.LIGHT, 0.14),), maxeval=4096,
                       precision="fp64")
    dip = gbw_obj()
    Q2s = torch.tensor([2.0, 10.0, 40.0], dtype=torch.float64)
    xs = torch.tensor([1e-3, 3e-4, 1e-2], dtype=torch.float64)
    batch = structure_functions(Q2s, xs, dip, config, seed=3)
    for i in range(3):
        alone = F2(Q2s[i].cuda(), xs[i].cuda(), dip, config, seed=3)
        assert float(batch["F2"][i]) == pytest.approx(float(alone.value), rel=1e-12)
        assert float(batch["F2_error"][i]) == pytest.approx(float(alone.error), rel=1e-9)


def test_vegas_is_deterministic():
    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.dis.observables import kinematics
    from nlo_bk_optimized_b200.numerics.integration import VegasOptions, vegas_terms

    config, quark, Q2, xbj, transverse = config_of("light_T_bk")
    kin = kinematics(Q2, xbj, pol_of(transverse), config, quark)
    dip = table_obj()
    opts = VegasOptions(samples_per_iteration=1 << 14, max_iterations=4, min_iterations=4, bins=50, epsrel=1e-12)
    a = vegas_terms(_native.DIS_TERMS["I1"], [kin], dip.native(), opts, [0], precision=_native.PRECISION_MIXED,
                    device=torch.device("cuda"))
    b = vegas_terms(_native.DIS_TERMS["I1"], [kin], dip.native(), opts, [0], precision=_native.PRECISION_MIXED,
                    device=torch.device("cuda"))
    assert torch.equal(a, b)


# ----------------------------------------------------------------------------- fixed-Sobol qqbar-g path


def _fixed_points(dims, seed, n):
    return torch.quasirandom.SobolEngine(dims, scramble=True, seed=seed).draw_base2(
        int(math.log2(n)), dtype=torch.float32).double().numpy()


@pytest.mark.parametrize("transverse", [True, False])
def test_fixed_sobol_matches_oracle(transverse):
    """Device fixed-Sobol flow (FP64) against the oracle's restatement on the same points:
    grid after training and every replicate estimate."""
    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.dis import DISConfig, Quark, QuarkType
    from nlo_bk_optimized_b200.dis.fixed_sobol import fixed_sobol_device

    config = DISConfig(quarks=(Quark(QuarkType.C, 1.4),), maxr=5.0, nf_alphas=1)
    dip = gbw_obj()
    Q2, xbj, seed = 9.0, 1e-3, 21
    nt, rounds, nr, reps = 1024, 2, 512, 3
    grid, est = fixed_sobol_device(Q2, xbj, pol_of(transverse), config.quarks[0], dip, config, seed=seed,
                                   device=torch.device("cuda"), precision=_native.PRECISION_FP64,
                                   training_samples=nt, training_rounds=rounds, samples_per_replicate=nr,
                                   replicates=reps)
    q, lam, g, x0 = GOLDEN["gbw_params"]
    odip = od.GBWDipole(qs0sqr=q, lam=lam, gamma=g, x0=x0)
    okin = od.Kinematics(Q2=Q2, xbj=xbj, mf=1.4, transverse=transverse, maxr=5.0, active_flavors=1)
    training = [_fixed_points(5, seed + r, nt) for r in range(rounds)]
    replicates = [_fixed_points(5, seed + 10_000 + j, nr) for j in range(reps)]
    edges, ref = od.fixed_sobol(lambda x: od.qg_triple(x, okin, odip), training, replicates, 5.0, bins=32)
    got_edges = grid[: 5 * 33].reshape(5, 33).cpu().numpy()
    assert np.max(np.abs(got_edges - edges)) < 1e-10
    assert rel_err(est.cpu().numpy(), ref) < 1e-9


REFERENCE_CPP = {  # T/benchmarks/dis_fixed_sobol_all_qg.py:69-76: (value, standard error)
    ("L", 0): (0.10206739088678346, 0.0002535000977528945),
    ("L", 1): (-0.024439455902300525, 0.00004764427185133986),
    ("L", 2): (0.009414936380564324, 0.000026852425497947778),
    ("T", 0): (0.40263591173620866, 0.0017956984452001683),
    ("T", 1): (-0.08719375357937224, 0.00026850014906050766),
    ("T", 2): (0.04848797141670969, 0.00013338145018266037),
}


@pytest.mark.parametrize("transverse", [True, False])
def test_fixed_sobol_agrees_with_reference_cpp_values(transverse):
    """Statistical pin: the GBW charm workload of the reference's fixed-Sobol benchmark
    (GBW(1, 0.3, 1, 1), m = 1.4, Q^2 = 9, x = 1e-3, maxr = 5, nf = 1, seed 3100) against the
    C++ values it quotes; agreement within 5 combined standard errors."""
    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.dipole import GBW
    from nlo_bk_optimized_b200.dis import DISConfig, Quark, QuarkType
    from nlo_bk_optimized_b200.dis.fixed_sobol import fixed_sobol_device

    config = DISConfig(quarks=(Quark(QuarkType.C, 1.4),), maxr=5.0, nf_alphas=1, epsrel=0.001)
    dip = GBW(Qs0sqr=1.0, lambda_=0.3, gamma=1.0, x0=1.0)
    _, est = fixed_sobol_device(9.0, 1e-3, pol_of(transverse), config.quarks[0], dip, config, seed=3100,
                                device=torch.device("cuda"), precision=_native.PRECISION_MIXED)
    est = est.cpu().numpy()
    tag = "T" if transverse else "L"
    for k in range(3):
        value, err = od.replicate_result(est[:, k])
        ref, ref_err = REFERENCE_CPP[(tag, k)]
        assert abs(value - ref) <= 5 * math.hypot(err, ref_err), (tag, k, value, err, ref, ref_err)


def test_sigma_qg_dispatches_by_precision():
    """float32 kinematics with GBW take the fixed-Sobol path (FIXED_SOBOL_EVALUATIONS
    evaluations per quark); float64 takes Vegas."""
    from nlo_bk_optimized_b200.dipole import GBW
    from nlo_bk_optimized_b200.dis import FIXED_SOBOL_EVALUATIONS, DISConfig, Polarization, Quark, QuarkType
    from nlo_bk_optimized_b200.dis import sigma_qg_d2b

    config = DISConfig(quarks=(Quark(QuarkType.C, 1.4),), maxr=5.0, nf_alphas=1, epsrel=0.05)
    dip = GBW(Qs0sqr=1.0, lambda_=0.3, gamma=1.0, x0=1.0)
    r32 = sigma_qg_d2b(torch.tensor(9.0, device="cuda"), torch.tensor(1e-3, device="cuda"), Polarization.L, dip,
                       config, seed=0)
    assert r32.n_eval == FIXED_SOBOL_EVALUATIONS
    small = DISConfig(quarks=config.quarks, maxr=5.0, nf_alphas=1, epsrel=0.05, maxeval=20_000)
    r64 = sigma_qg_d2b(torch.tensor(9.0, dtype=torch.float64, device="cuda"),
                       torch.tensor(1e-3, dtype=torch.float64, device="cuda"), Polarization.L, dip, small, seed=0)
    assert r64.n_eval != FIXED_SOBOL_EVALUATIONS
    diff = abs(float(r64.value) - float(r32.value))
    assert diff <= 5 * math.hypot(float(r64.error), float(r32.error)) + 0.02 * abs(float(r32.value))
