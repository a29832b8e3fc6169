"""Host tests of the nlo-bk / nlo-dis command lines (cli/nlobk.py, cli/nlodis.py of the
reference): options, defaults, the configurations they build and the argument errors."""

from __future__ import annotations

import math

import pytest
import torch

from nlo_bk_optimized_b200.bk.config import (
    BKOrder,
    IntegrationMethod,
    ResummationCoupling,
    RunningCouplingLO,
    RunningCouplingNLO,
    device_supported,
)
from nlo_bk_optimized_b200.cli import nlobk, nlodis
from nlo_bk_optimized_b200.dis.config import DISOrder, QuarkType, RunningCouplingIRScheme, RunningCouplingScheme


def test_nlobk_defaults_build_a_device_configuration():
    args = nlobk._parser().parse_args([])
    assert (args.x0, args.qs0sqr, args.gamma, args.ec, args.lambdaqcd) == (0.01, 0.10, 1.0, 1.0, 0.241)
    assert (args.maxy, args.output, args.nf, args.C2, args.fixed_alpha_s, args.Ksub) == (10.0, "output.dat", 3, 1.0,
                                                                                         0.2, 0.65)
    assert (args.minr, args.maxr, args.rpoints, args.mcintpoints, args.step) == (1e-6, 30.0, 100, 100_000, 0.2)
    assert args.device == "cuda" and args.dtype == "float32" and args.seed is None
    config = nlobk.config_from_args(args)
    assert config.Order is BKOrder.NLO_RESUM_DLOG_SLOG
    assert config.RC_LO is RunningCouplingLO.BALITSKY_LO and config.RC_NLO is RunningCouplingNLO.SMALLEST_NLO
    assert config.RESUM_RC is ResummationCoupling.RESUM_RC_SMALLEST
    assert config.INTMETHOD_NLO is IntegrationMethod.VEGAS  # the reference's default
    assert config.FORCE_POSITIVE_N and not config.DNDY and not config.EULER_METHOD
    assert (config.RPOINTS, config.MINR, config.MAXR, config.MCINTPOINTS) == (100, 1e-6, 30.0, 100_000)
    assert device_supported(config) is None


def test_nlobk_option_mapping():
    args = nlobk._parser().parse_args(["--rc-lo", "fixed", "--rc-nlo", "parent", "--nolimit", "--dndy", "--euler",
                                       "--nf", "0", "--C2", "2.5", "--fixed-alpha-s", "0.15", "--Ksub", "0.5"])
    config = nlobk.config_from_args(args)
    # a fixed LO coupling fixes the NLO coupling (cli/nlobk.py:40, 51)
    assert config.RC_LO is RunningCouplingLO.FIXED_LO and config.RC_NLO is RunningCouplingNLO.FIXED_NLO
    assert not config.FORCE_POSITIVE_N and config.DNDY and config.EULER_METHOD and config.stepper == "euler"
    assert (config.NF, config.C2, config.FIXED_AS, config.KSUB) == (0, 2.5, 0.15, 0.5)
    assert device_supported(config) is None


@pytest.mark.parametrize("argv,why", [
    (["--integration", "miser"], "MISER"),
    (["--integration", "multiple"], "MULTIPLE"),
])
def test_nlobk_switches_outside_the_device_kernels(argv, why):
    config = nlobk.config_from_args(nlobk._parser().parse_args(argv))
    assert why in device_supported(config)


@pytest.mark.parametrize("argv", [
    ["--order", "lo"], ["--order", "nlo"], ["--order", "lo_resum_dlog"], ["--order", "nlo_resum_dlog"],
    ["--rc-lo", "parent"], ["--rc-lo", "smallest"], ["--rc-lo", "fac"], ["--rc-lo", "beuf"],
    ["--resum-rc", "fixed"], ["--resum-rc", "parent"], ["--rc-nlo", "parent"], ["--nf", "5"], ["--nf", "0"],
    ["--kinematical-constraint", "--euler"], ["--integration", "sobol", "--order", "nlo"],
    # orders without NLO kernels never integrate K2 + Kf, so its method does not matter
    ["--order", "lo", "--integration", "miser"],
])
def test_nlobk_variants_run_on_the_device(argv):
    from nlo_bk_optimized_b200.bk.evolution import params_of

    config = nlobk.config_from_args(nlobk._parser().parse_args(argv))
    assert device_supported(config) is None
    params = params_of(config, 0)
    switches = (params.order, params.rc_lo, params.resum_rc, params.rc_nlo, params.kinematical_constraint)
    assert switches != (0, 0, 0, 0, 0) or argv in (["--nf", "5"], ["--nf", "0"])


def test_nlobk_argument_errors(capsys):
    with pytest.raises(SystemExit) as stop:
        nlobk.main(["--device", "cpu"])
    assert stop.value.code == 2
    assert "CUDA" in capsys.readouterr().err
    with pytest.raises(SystemExit):
        nlobk._parser().parse_args(["--integration", "quad"])
    # the kinematical constraint needs the Euler stepper, as in the reference's BKConfig
    with pytest.raises(ValueError):
        nlobk.config_from_args(nlobk._parser().parse_args(["--kinematical-constraint"]))


def test_nlodis_options_and_configuration():
    argv = ["--datafile", "t.dat", "--C2", "7.2", "--charm-mass", "1.35", "--proton-area", "8.5", "--rc-scheme",
            "PARENT"]
    args = nlodis._parser().parse_args(argv)
    assert (args.name, args.light_mass, args.order, args.runmode, args.epsrel) == ("nlodis", 0.01, "NLO", "HERA_FL",
                                                                                   0.01)
    assert (args.mcintpoints, args.nf, args.maxr, args.quadrature_points, args.batch_size) == (1_000_000, -1, 30.0,
                                                                                                24, 65_536)
    assert (args.seed, args.device, args.dtype, args.cuda_nested_points) == (0, "cuda", "float32", 48)
    config = nlodis.config_from_args(args)
    assert config.order is DISOrder.NLO and config.rc_scheme is RunningCouplingScheme.PARENT
    assert config.rc_ir_scheme is RunningCouplingIRScheme.SMOOTH
    assert config.transverse_area == pytest.approx(8.5 * 2.56819, rel=1e-15)
    assert [q.type for q in config.quarks] == [QuarkType.LIGHT, QuarkType.C]
    assert [q.mass for q in config.quarks] == [0.01, 1.35]
    assert (config.C2_alpha, config.nf_alphas, config.maxeval, config.epsrel) == (7.2, -1, 1_000_000, 0.01)
    assert config.precision == "mixed"
    args = nlodis._parser().parse_args([*argv, "--dtype", "float64", "--order", "LO"])
    config = nlodis.config_from_args(args)
    assert config.precision == "fp64" and config.order is DISOrder.LO
    for missing in ("--datafile", "--C2", "--charm-mass", "--proton-area", "--rc-scheme"):
        i = argv.index(missing)
        with pytest.raises(SystemExit):
            nlodis._parser().parse_args(argv[:i] + argv[i + 2:])


def test_nlodis_points():
    assert len(nlodis.HERA_FL_POINTS) == 20
    assert nlodis.HERA_FL_POINTS[0] == (1.5, 0.000028) and nlodis.HERA_FL_POINTS[-1] == (346.0, 0.009860)
    grid = nlodis.grid_points()
    per_Q2 = math.floor(math.log(1e3) / math.log(1.5)) + 1  # 1e-5 * 1.5^k <= 1e-2
    assert len(grid) == 3 * per_Q2
    assert [q for q, _ in grid[::per_Q2]] == [4.5, 45.0, 100.0]
    assert grid[0][1] == 1e-5 and grid[per_Q2 - 1][1] <= 1e-2 < grid[per_Q2 - 1][1] * 1.5


@pytest.mark.parametrize("dtype,tol", [(torch.float32, 5e-9), (torch.float64, 1e-13)])
def test_legacy_table_round_trip_of_evolution_grids(tmp_path, dtype, tol):
    """solve_bk's grid (float64, rounded once for float32 tables) survives the legacy
    format: the header multiplier reproduces every r."""
    from nlo_bk_optimized_b200.bk.config import BKConfig
    from nlo_bk_optimized_b200.bk.evolution import _r_grid
    from nlo_bk_optimized_b200.dipole.table import DipoleTable, load_bk_table, save_bk_table

    r = _r_grid(BKConfig(RPOINTS=100, MINR=1e-6, MAXR=30.0), device="cpu", dtype=torch.float64)
    N = torch.linspace(0, 1, 202, dtype=torch.float64).reshape(2, 101)
    table = DipoleTable(r=r.to(dtype), y=torch.tensor([0.0, 0.2], dtype=dtype), N=N.to(dtype), x0=0.01)
    save_bk_table(tmp_path / "t.dat", table)
    back = load_bk_table(tmp_path / "t.dat")
    assert float((back.r / r - 1).abs().max()) < tol
    # 16 significant digits in the file: N comes back within 1e-15
    assert torch.allclose(back.N, N.to(dtype).double(), rtol=1e-15, atol=1e-300) and back.x0 == 0.01
