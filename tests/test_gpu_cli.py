"""The nlo-bk / nlo-dis command lines end to end on the device: --dndy against
compute_dndy, a table written and read back in the legacy format, LO HERA F_L from that
table against the oracle (LINEAR_LINEAR interpolation), and batched NLO F_L against the
same point run alone."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from oracle import dis as od

pytestmark = pytest.mark.gpu

BK_ARGS = ["--rpoints", "100", "--mcintpoints", "8192", "--seed", "1", "--step", "0.2"]
DIS_ARGS = ["--C2", "7.2", "--charm-mass", "1.35", "--proton-area", "8.5", "--rc-scheme", "SMALLEST"]


@pytest.fixture(scope="module")
def bk_table(tmp_path_factory):
    from nlo_bk_optimized_b200.cli import nlobk

    path = tmp_path_factory.mktemp("cli") / "bk.dat"
    assert nlobk.main([*BK_ARGS, "--maxy", "7.0", "--output", str(path)]) == 0
    return path


def test_nlobk_dndy_matches_compute_dndy(capsys):
    from nlo_bk_optimized_b200.bk import MV, compute_dndy
    from nlo_bk_optimized_b200.cli import nlobk

    assert nlobk.main([*BK_ARGS, "--dndy", "--rpoints", "60"]) == 0
    out = capsys.readouterr().out.splitlines()
    assert out[0] == "# r dN/dy[K1] dN/dy[K2+Kf] N"
    rows = np.array([[float(v) for v in line.split()] for line in out[1:]])
    config = nlobk.config_from_args(nlobk._parser().parse_args([*BK_ARGS, "--dndy", "--rpoints", "60"]))
    ref = compute_dndy(MV(qs0sqr=0.10, x0=0.01), config, device="cuda", dtype=torch.float32, seed=1)
    want = torch.stack((ref.r, ref.K1, ref.K2_Kf, ref.N), dim=1).double().cpu().numpy()
    assert rows.shape == want.shape and rows.shape[0] > 10
    np.testing.assert_allclose(rows, want, rtol=1e-14, atol=0)


def test_nlobk_writes_the_legacy_table(bk_table, capsys):
    from nlo_bk_optimized_b200.dipole import load_bk_table

    table = load_bk_table(bk_table)
    assert table.r.numel() == 101 and table.y.numel() == 36
    assert table.x0 == pytest.approx(0.01)
    assert float(table.y[-1]) == pytest.approx(7.0, rel=1e-12)
    N = table.N.numpy()
    assert np.all(np.isfinite(N)) and np.all(N >= 0) and np.all(N <= 1)
    mid = (N[0] > 0.01) & (N[0] < 0.9)  # away from the frozen, saturated parents and tiny N
    assert mid.sum() > 10 and np.all(N[-1][mid] > N[0][mid])  # the amplitude grows with rapidity


def _printed(out: str) -> list[list[str]]:
    return [line.split(",") for line in out.splitlines() if line and not line.startswith("fit,")]


@pytest.mark.parametrize("dtype,tol", [("float64", 1e-11), ("float32", 1e-4)])
def test_nlodis_lo_hera_fl_matches_oracle(bk_table, capsys, dtype, tol):
    from nlo_bk_optimized_b200.cli import nlodis
    from nlo_bk_optimized_b200.dipole import load_bk_table

    assert nlodis.main(["--datafile", str(bk_table), *DIS_ARGS, "--order", "LO", "--dtype", dtype]) == 0
    captured = capsys.readouterr()
    assert captured.out.splitlines()[0] == "fit,x,Q2,FL"
    rows = _printed(captured.out)
    assert len(rows) == 20 and all(r[0] == "nlodis" for r in rows)
    assert captured.err.count("# FL Q2=") == 20
    table = load_bk_table(bk_table)
    dip = od.TableDipole(table.r.numpy(), table.y.numpy(), table.N.numpy(), x0=table.x0,
                         interpolation="linear_linear")
    quarks = [(0.01, 2 / 3), (1.35, 4 / 9)]
    area = 8.5 * nlodis.MB_TO_GEV2
    for (Q2, x), row in zip(nlodis.HERA_FL_POINTS, rows):
        assert (float(row[1]), float(row[2])) == (x, Q2)
        dip.initialize(max(math.log(dip.X0() / x), 0.0))
        sigma = od.LO_FACTOR * od.gauss_legendre_tensor(
            lambda u: od.lo_integrand(u, Q2, x, quarks, False, dip), 2, 24)
        assert float(row[3]) == pytest.approx(sigma * od.structure_function_factor(Q2, area), rel=tol)


def test_nlodis_nlo_batch_equals_points_alone(bk_table):
    """The command line's batched NLO run gives each point's FL(...) run alone."""
    from dataclasses import replace

    from nlo_bk_optimized_b200.cli import nlodis
    from nlo_bk_optimized_b200.dipole import AmplitudeInterpolation, BKDipole, load_bk_table
    from nlo_bk_optimized_b200.dis import FL, Polarization, structure_function_batch

    args = nlodis._parser().parse_args(["--datafile", str(bk_table), *DIS_ARGS, "--mcintpoints", "4096",
                                        "--dtype", "float64"])
    config = replace(nlodis.config_from_args(args), quarks=nlodis.config_from_args(args).quarks[:1])
    table = load_bk_table(bk_table, device="cuda")
    dipole = BKDipole(table, interpolation=AmplitudeInterpolation.LINEAR_LINEAR)
    points = nlodis.HERA_FL_POINTS[::7]
    batch = structure_function_batch([(Q2, x, Polarization.L, 5) for Q2, x in points], dipole, config)
    for (Q2, x), got in zip(points, batch):
        alone = FL(torch.tensor(Q2, dtype=torch.float64, device="cuda"),
                   torch.tensor(x, dtype=torch.float64, device="cuda"), dipole, config, seed=5)
        assert float(got.value) == pytest.approx(float(alone.value), rel=1e-12)
        assert float(got.error) == pytest.approx(float(alone.error), rel=1e-9)
        assert got.n_eval == alone.n_eval and math.isfinite(float(got.value))


def test_nlodis_lo_grid_is_additive_in_quarks(bk_table, capsys):
    """F2FL_GRID at LO: F_2 is linear in the quark sum, so F2 light + F2 charm = F2_LO,
    and the light F_L of the first grid point matches the oracle."""
    from nlo_bk_optimized_b200.cli import nlodis
    from nlo_bk_optimized_b200.dipole import load_bk_table

    assert nlodis.main(["--datafile", str(bk_table), *DIS_ARGS, "--order", "LO", "--runmode", "F2FL_GRID",
                        "--dtype", "float64", "--no-header"]) == 0
    captured = capsys.readouterr()
    rows = _printed(captured.out)
    grid = nlodis.grid_points()
    assert len(rows) == len(grid)
    assert captured.err.count("# FT_light") == len(grid) and captured.err.count("# FL_charm") == len(grid)
    for row in rows:
        F2l, F2c, F2lo = float(row[3]), float(row[5]), float(row[7])
        assert F2l + F2c == pytest.approx(F2lo, rel=1e-12)
    table = load_bk_table(bk_table)
    dip = od.TableDipole(table.r.numpy(), table.y.numpy(), table.N.numpy(), x0=table.x0,
                         interpolation="linear_linear")
    Q2, x = grid[0]
    dip.initialize(max(math.log(dip.X0() / x), 0.0))
    sigma = od.LO_FACTOR * od.gauss_legendre_tensor(
        lambda u: od.lo_integrand(u, Q2, x, [(0.01, 2 / 3)], False, dip), 2, 24)
    assert float(rows[0][4]) == pytest.approx(sigma * od.structure_function_factor(Q2, 8.5 * nlodis.MB_TO_GEV2),
                                              rel=1e-11)
