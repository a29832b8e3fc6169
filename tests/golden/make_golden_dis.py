"""Generate ``dis_reference.npz`` from the reference implementation's DIS path.

Run with the root of a reference checkout (read-only is enough) in the environment
variable ``NLO_REFERENCE_ROOT`` (or as the first argument)::

    NLO_REFERENCE_ROOT=<checkout> python tests/golden/make_golden_dis.py [<checkout>]

The script puts ``<checkout>/torch_nlo_clean/src`` on the import path itself.

It imports the reference package ``nlo_torch`` and records, in float64 on the CPU,
what its own functions return for seeded inputs:

* a synthetic BK table (MV-shaped rows, saturation scale growing with Y) and the
  reference ``BKDipole`` amplitude on it, both the local 7/9-point spline path and the
  initialised global spline (dipole/amplitude.py:48-252);
* the GBW amplitude (dipole/amplitude.py:23-45) and the DIS couplings (coupling.py:49-97);
* ``Li2`` and the Bessel functions the DIS code calls (numerics/special.py:10-96);
* the LO integrand with its radial Jacobian (dis/lo.py:12-51, dis/observables.py:352-359)
  and the LO cross section by the tensor Gauss-Legendre rule (dis/observables.py:334-384);
* ``integrand_dip_massive`` for T0/T1/T2 and Omega_L/ab/cd (dis/observables.py:107-172);
* ``integrand_qgunsub_massive`` for I1 (5D), I2 (6D) and I3 (7D) (dis/observables.py:175-250);
* one ``vegas`` run on a dipole term (numerics/integration.py:120-589) with its final grid;
* LO-order F_T, F_L, F_2 (dis/observables.py:581-624);
* the fixed-Sobol sampling pieces ``map_importance_grid`` and ``paired_endpoint_inputs``
  (dis/fixed_sobol.py:100-158) and one ``_adapt_vegas_edges`` re-binning
  (numerics/integration.py:804-866) on float64 inputs;
* the LINEAR_LINEAR table interpolation (dipole/amplitude.py:188-212): amplitudes on the
  local and the initialised path, one dipole term and LO F_T, F_L with it.

Unit-cube points come from numpy's default_rng(20260301); each case is listed in
``cases`` with its kinematics.
"""

from __future__ import annotations

import math
import os
import sys
from pathlib import Path

import numpy as np
import torch

_ROOT = next((a for a in reversed(sys.argv[1:]) if Path(a).is_dir()), os.environ.get("NLO_REFERENCE_ROOT"))
if not _ROOT:
    raise SystemExit("set NLO_REFERENCE_ROOT (or pass the checkout) to the reference checkout's root")
sys.path.insert(0, str(Path(_ROOT) / "torch_nlo_clean" / "src"))

from nlo_torch.coupling import dis_alpha_s_freeze, dis_alpha_s_smooth
from nlo_torch.dipole.amplitude import GBW, BKDipole
from nlo_torch.dipole.table import DipoleTable
from nlo_torch.dis.config import (
    DISConfig,
    NcScheme,
    Polarization,
    Quark,
    QuarkType,
    RunningCouplingIRScheme,
    RunningCouplingScheme,
)
from nlo_torch.dis.lo import integrand_photon_target_LO
from nlo_torch.dis.observables import (
    F2,
    FL,
    FT,
    integrand_dip_massive,
    integrand_qgunsub_massive,
    photon_proton_cross_section_LO_d2b,
)
from nlo_torch.numerics.integration import vegas
from nlo_torch.numerics.special import Li2, bessel_K0, bessel_K1

torch.set_default_dtype(torch.float64)
OUT = Path(__file__).with_name("dis_reference.npz")
T64 = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float64)  # noqa: E731


def synthetic_table():
    """120 log-spaced r in [1e-6, 50], Y = 0, 0.5, ..., 14; MV rows with Qs^2 = 0.2 e^{0.3 Y}."""
    r = 1e-6 * (50 / 1e-6) ** (np.arange(120) / 119)
    y = np.arange(29) * 0.5
    qs2 = 0.2 * np.exp(0.3 * y)[:, None]
    N = 1 - np.exp(-(r[None, :] ** 2 * qs2 / 4) * np.log(1 / (r[None, :] * 0.241) + math.e))
    return r, y, N


def main() -> None:
    rng = np.random.default_rng(20260301)
    out: dict[str, np.ndarray] = {}
    r_tab, y_tab, N_tab = synthetic_table()
    out["table_r"], out["table_y"], out["table_N"] = r_tab, y_tab, N_tab
    table = DipoleTable(T64(r_tab), T64(y_tab), T64(N_tab), 1.0)

    # amplitudes: local path on scattered (r, Y), then the initialised spline at Y = 4.7
    amp_r = np.exp(rng.uniform(math.log(5e-7), math.log(80.0), 400))
    amp_Y = rng.uniform(0.0, 14.0, 400)
    bk = BKDipole(table)
    out["amp_r"], out["amp_Y"] = amp_r, amp_Y
    out["amp_local"] = bk.dipole_amplitude(T64(amp_r), T64(amp_Y)).numpy()
    bk.initialize_interpolation(4.7)
    out["amp_init_Y"] = np.array([4.7])
    out["amp_init"] = bk.dipole_amplitude(T64(amp_r), torch.full((400,), 4.7)).numpy()
    out["amp_init_maxr"] = np.array([bk.maxr_interpolate])
    gbw = GBW(Qs0sqr=0.25, lambda_=0.29, gamma=1.1, x0=0.01)
    out["gbw_params"] = np.array([0.25, 0.29, 1.1, 0.01])
    out["gbw"] = gbw.dipole_amplitude(T64(amp_r), T64(amp_Y)).numpy()

    # special functions and couplings
    li_x = np.concatenate([rng.uniform(-30, 1, 300), [-1.0, 0.0, 0.5, 1.0, -1e-8, 0.49999]])
    out["li2_x"], out["li2"] = li_x, Li2(T64(li_x)).numpy()
    bx = np.exp(rng.uniform(math.log(1e-7), math.log(500), 300))
    out["bessel_x"], out["k0"], out["k1"] = bx, bessel_K0(T64(bx)).numpy(), bessel_K1(T64(bx)).numpy()
    ar = np.exp(rng.uniform(math.log(1e-6), math.log(100), 200))
    out["alpha_r"] = ar
    out["alpha_freeze"] = dis_alpha_s_freeze(T64(ar), Nf=3, C2=1.0, max_alpha_s=0.7).numpy()
    out["alpha_smooth"] = dis_alpha_s_smooth(T64(ar), Nf=4, C2=2.0).numpy()

    light = Quark(QuarkType.LIGHT, 0.14)
    charm = Quark(QuarkType.C, 1.4)
    cases = [
        # name, Q2, xbj, quark, pol, dipole kind, config overrides
        ("light_T_bk", 10.0, 1e-3, light, Polarization.T, "bk", {}),
        ("light_L_bk", 10.0, 1e-3, light, Polarization.L, "bk", {}),
        ("charm_T_gbw", 25.0, 3e-4, charm, Polarization.T, "gbw", {}),
        ("charm_L_gbw", 25.0, 3e-4, charm, Polarization.L, "gbw", {}),
        ("light_T_gbw_smooth_parent", 3.0, 1e-2, light, Polarization.T, "gbw",
         {"rc_ir_scheme": RunningCouplingIRScheme.SMOOTH, "rc_scheme": RunningCouplingScheme.PARENT,
          "nc_scheme": NcScheme.LargeNC}),
        ("light_L_bk_lowQ", 1.5, 5e-5, light, Polarization.L, "bk", {"maxr": 25.0}),
    ]
    names = []
    for name, Q2v, xv, quark, pol, kind, over in cases:
        names.append(name)
        config = DISConfig(quarks=(quark,), cuda_fusion=False, cuda_nested=False, **over)
        Q2 = torch.tensor(Q2v)
        xbj = torch.tensor(xv)
        dipole = BKDipole(table) if kind == "bk" else gbw
        out[f"{name}/kin"] = np.array([Q2v, xv, quark.mass, quark.charge**2, pol is Polarization.T,
                                       config.maxr, config.nc_scheme is NcScheme.FiniteNC,
                                       config.rc_scheme is RunningCouplingScheme.PARENT,
                                       config.rc_ir_scheme is RunningCouplingIRScheme.SMOOTH,
                                       config.C2_alpha, config.active_flavors, config.max_alpha_s_freeze],
                                      dtype=np.float64)
        # dipole terms (fresh BK dipole: the local spline path)
        for order, contribution in enumerate(("T0", "T1", "T2") if pol is Polarization.T
                                             else ("Omega_L_const", "ab", "cd")):
            x = rng.uniform(0, 1, (256, 2 + order))
            x[:4, 0] = [1e-7, 1 - 1e-7, 0.5, 0.999]
            out[f"{name}/dip{order}_x"] = x
            out[f"{name}/dip{order}"] = integrand_dip_massive(
                T64(x), Q2, xbj, pol, quark, contribution, dipole, config).numpy()
        for contribution, dims in (("I1", 5), ("I2", 6), ("I3", 7)):
            x = rng.uniform(0, 1, (256, dims))
            out[f"{name}/qg_{contribution}_x"] = x
            out[f"{name}/qg_{contribution}"] = integrand_qgunsub_massive(
                T64(x), Q2, xbj, pol, quark, contribution, dipole, config).numpy()
        # LO integrand (all quarks of the config) and LO cross section by Gauss-Legendre
        lo_dipole = BKDipole(table) if kind == "bk" else gbw
        Y = max(math.log(lo_dipole.X0() / xv), 0.0)
        if kind == "bk":
            lo_dipole.initialize_interpolation(Y)
        x = rng.uniform(0, 1, (256, 2))
        r = config.maxr * T64(x[:, 1])
        lo = 2 * math.pi * r * config.maxr * integrand_photon_target_LO(
            r, T64(x[:, 0]), xbj, Q2, pol, config.quarks, lo_dipole)
        out[f"{name}/lo_x"], out[f"{name}/lo"] = x, lo.numpy()
        res = photon_proton_cross_section_LO_d2b(Q2, xbj, pol, lo_dipole, config)
        out[f"{name}/sigma_lo"] = np.array([float(res.value), float(res.error)])

    # Vegas pin: T1 dipole term of the first case, 3 iterations x 3000 samples, 50 bins
    config = DISConfig(quarks=(light,), cuda_fusion=False, cuda_nested=False)
    fn = lambda x: integrand_dip_massive(  # noqa: E731
        x, torch.tensor(10.0), torch.tensor(1e-3), Polarization.T, light, "T1", gbw, config)
    from nlo_torch.numerics.integration import VegasState

    state = VegasState()
    res = vegas(fn, torch.tensor([[0.0, 1.0]] * 3), samples_per_iteration=3000, max_iterations=3,
                min_iterations=3, bins=50, batch_size=1 << 20, epsrel=1e-9, seed=7, state=state)
    out["vegas_pin"] = np.array([float(res.value), float(res.error), res.n_eval, res.converged, 7, 3000, 3, 50])
    out["vegas_pin_edges"] = state.edges.numpy()

    # LO-order structure functions (GBW and BK)
    for kind in ("gbw", "bk"):
        config = DISConfig(quarks=(Quark(QuarkType.LIGHT, 0.14), Quark(QuarkType.C, 1.4)),
                           cuda_fusion=False, cuda_nested=False)
        dip = gbw if kind == "gbw" else BKDipole(table)
        Q2, xbj = torch.tensor(7.5), torch.tensor(2e-4)
        out[f"lo_sf_{kind}"] = np.array([float(FT(Q2, xbj, dip, config).value),
                                         float(FL(Q2, xbj, dip, config).value),
                                         float(F2(Q2, xbj, dip, config).value)])
    # fixed-Sobol sampling pieces (dis/fixed_sobol.py:100-158) and the grid re-binning
    # (numerics/integration.py:804-866) on float64 inputs, with their own generator
    from nlo_torch.dis.fixed_sobol import map_importance_grid, paired_endpoint_inputs
    from nlo_torch.numerics.integration import _adapt_vegas_edges

    frng = np.random.default_rng(777)
    fs_points = frng.uniform(0, 1, (256, 5))
    widths = frng.uniform(0.2, 1.0, (5, 32))
    fs_edges = np.concatenate([np.zeros((5, 1)), np.cumsum(widths, axis=1) / widths.sum(axis=1, keepdims=True)],
                              axis=1)
    fs_edges[:, -1] = 1.0
    src, inv, bi = map_importance_grid(T64(fs_points), T64(fs_edges))
    out["fs_points"], out["fs_edges"] = fs_points, fs_edges
    out["fs_source"], out["fs_inv"], out["fs_bins"] = src.numpy(), inv.numpy(), bi.numpy()
    for fold in (False, True):
        f, fw, sc, sw = paired_endpoint_inputs(src, 5.0, fold_angle=fold)
        tag = "fold" if fold else "nofold"
        out[f"fs_first_{tag}"], out[f"fs_fw_{tag}"] = f.numpy(), fw.numpy()
        out[f"fs_second_{tag}"], out[f"fs_sw_{tag}"] = sc.numpy(), sw.numpy()
    hist = frng.uniform(0, 3, (5, 32))
    count = frng.integers(0, 9, (5, 32)).astype(np.float64)
    out["adapt_hist"], out["adapt_count"] = hist, count
    out["adapt_edges"] = _adapt_vegas_edges(T64(fs_edges), T64(hist), T64(count), cuda_fusion=False).numpy()
    # LINEAR_LINEAR table interpolation (dipole/amplitude.py:188-212), with its own
    # generator: scattered (r, Y) plus the edges (r outside the table, on a knot and on the
    # last knot; Y on a row and on the last row), the initialised spline, one dipole term
    # and the LO structure functions
    from nlo_torch.dipole.amplitude import AmplitudeInterpolation

    brng = np.random.default_rng(4242)
    b_r = np.concatenate([np.exp(brng.uniform(math.log(5e-7), math.log(80.0), 300)),
                          [r_tab[0] * 0.5, r_tab[-1] * 2, r_tab[-1], r_tab[17], r_tab[0], 1.0, 3.0]])
    b_Y = np.concatenate([brng.uniform(0.0, 14.0, 300), [3.0, 14.0, 14.0, 5.5, 0.0, 14.0, 7.25]])
    linear = BKDipole(table, interpolation=AmplitudeInterpolation.LINEAR_LINEAR)
    out["bilin_r"], out["bilin_Y"] = b_r, b_Y
    out["bilin_amp"] = linear.dipole_amplitude(T64(b_r), T64(b_Y)).numpy()
    linear.initialize_interpolation(4.7)
    out["bilin_init"] = linear.dipole_amplitude(T64(b_r), torch.full((b_r.size,), 4.7)).numpy()
    out["bilin_init_maxr"] = np.array([linear.maxr_interpolate])
    config = DISConfig(quarks=(light,), cuda_fusion=False, cuda_nested=False)
    x = brng.uniform(0, 1, (256, 3))
    linear = BKDipole(table, interpolation=AmplitudeInterpolation.LINEAR_LINEAR)
    out["bilin_dip1_x"] = x
    out["bilin_dip1"] = integrand_dip_massive(T64(x), torch.tensor(10.0), torch.tensor(1e-3), Polarization.T,
                                              light, "T1", linear, config).numpy()
    config = DISConfig(quarks=(Quark(QuarkType.LIGHT, 0.14), Quark(QuarkType.C, 1.4)),
                       cuda_fusion=False, cuda_nested=False)
    Q2, xbj = torch.tensor(7.5), torch.tensor(2e-4)
    out["bilin_lo_sf"] = np.array([
        float(FT(Q2, xbj, BKDipole(table, interpolation=AmplitudeInterpolation.LINEAR_LINEAR), config).value),
        float(FL(Q2, xbj, BKDipole(table, interpolation=AmplitudeInterpolation.LINEAR_LINEAR), config).value)])

    out["cases"] = np.array(names)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()
