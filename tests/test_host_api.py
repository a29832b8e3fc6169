"""Host-side behaviour that needs no GPU: configuration, table I/O, stepping
counts, initial conditions, and the C-ABI library's exports."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest
import torch

from golden_data import bk_table_mc50w
from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.bk.config import BKConfig, IntegrationMethod, RunningCouplingLO, device_supported
from nlo_bk_optimized_b200.bk.evolution import _r_grid, _steps_to, nlo_box, solve_bk
from nlo_bk_optimized_b200.bk.initial_conditions import MV, ICDataFile
from nlo_bk_optimized_b200.dipole.table import DipoleTable, load_bk_table, save_bk_table

ROOT = Path(__file__).resolve().parent.parent


def test_config_defaults_and_validation():
    config = BKConfig()
    assert config.NC == 3.0 and config.NF == 3 and config.RPOINTS == 100
    # the reference's production path: Vegas per parent with grid reuse, Kutta RK3
    assert config.INTMETHOD_NLO is IntegrationMethod.VEGAS
    assert config.VEGAS_REUSE_GRID and config.VEGAS_REUSE_WARMUP_FRACTION == 0.25
    assert config.stepper == "rk3"
    assert BKConfig(EULER_METHOD=True).stepper == "euler"
    with pytest.raises(ValueError):
        BKConfig(NF=4)
    with pytest.raises(ValueError):
        BKConfig(MINR=1.0, MAXR=0.5)
    with pytest.raises(ValueError):
        BKConfig(RC_LO=RunningCouplingLO.FIXED_LO)  # needs FIXED_NLO too (bk/config.py:119-122)
    with pytest.raises(ValueError):
        BKConfig(STEPPER="rk45")
    with pytest.raises(ValueError):
        BKConfig(KINEMATICAL_CONSTRAINT=True)
    assert device_supported(config) is None
    assert device_supported(BKConfig(INTMETHOD_NLO=IntegrationMethod.SOBOL)) is None
    assert "MISER" in device_supported(BKConfig(INTMETHOD_NLO=IntegrationMethod.MISER))


def test_r_grid_matches_reference_construction():
    config = BKConfig(RPOINTS=399, MINR=1e-7, MAXR=1e2)
    r = _r_grid(config, device="cpu", dtype=torch.float64)
    assert r.numel() == 400
    assert r[0].item() == pytest.approx(1e-7, rel=1e-15)
    assert r[-1].item() == pytest.approx(1e2, rel=1e-12)
    lower, width = nlo_box(float(r[0]), float(r[-1]))
    assert lower[0] == pytest.approx(np.log(0.5e-7))
    assert lower[0] + width[0] == pytest.approx(np.log(200.0))
    assert width[2] == pytest.approx(2 * np.pi)


def test_step_count_follows_reference_accumulation():
    ys = _steps_to(0.0, 10.0, 0.1)
    assert len(ys) == 100
    assert ys[-1] == pytest.approx(10.0)
    assert len(_steps_to(0.0, 4.0, 0.2)) == 20
    assert len(_steps_to(0.0, 0.0, 0.2)) == 1  # the reference always takes one step


def test_cpu_device_is_rejected_without_fallback():
    with pytest.raises((ValueError, RuntimeError)):
        solve_bk(MV(qs0sqr=0.2), 0.2, BKConfig(RPOINTS=10), device="cpu")


def test_table_round_trip_and_legacy_format(tmp_path):
    golden = bk_table_mc50w()
    r = torch.tensor(golden["r"])
    table = DipoleTable(r=r, y=torch.tensor(golden["y"]), N=torch.tensor(golden["N"]), x0=float(golden["x0"][0]))
    path = tmp_path / "table.dat"
    save_bk_table(path, table)
    loaded = load_bk_table(path)
    torch.testing.assert_close(loaded.r, table.r, rtol=1e-14, atol=0)
    torch.testing.assert_close(loaded.y, table.y, rtol=0, atol=1e-15)
    torch.testing.assert_close(loaded.N, table.N, rtol=1e-14, atol=1e-300)
    assert loaded.x0 == table.x0
    # the C++ table: 101 r points from 1e-5, multiplier 1.16083692085089, x0 = 0.01
    assert r.numel() == 101 and r[0].item() == pytest.approx(1e-5)
    assert float(golden["x0"][0]) == pytest.approx(0.01)


def test_legacy_table_reader_rejects_malformed_files(tmp_path):
    grid = "###1e-5\n###1.5\n###3\n###0.01\n"
    cases = {
        "short_block": grid + "###0\n0.1\n0.2\n",
        "long_block": grid + "###0\n0.1\n0.2\n0.3\n0.4\n",
        "values_first": grid + "0.5\n###0\n0.1\n0.2\n0.3\n",
        "no_blocks": grid,
        "bad_value": grid + "###0\n0.1\nx\n0.3\n",
        "bad_grid": "###1e-5\n###0.5\n###3\n###0.01\n###0\n0.1\n0.2\n0.3\n",
        "three_directives": "###1e-5\n###1.5\n###3\n",
    }
    for name, text in cases.items():
        path = tmp_path / f"{name}.dat"
        path.write_text(text)
        with pytest.raises(ValueError):
            load_bk_table(path)
    good = tmp_path / "good.dat"
    good.write_text("# comment\n" + grid + "\n###0\n0.1\n0.2\n0.3\n## another comment\n###0.4\n0.2\n0.3\n0.4\n")
    table = load_bk_table(good)
    assert table.N.shape == (2, 3) and table.y.tolist() == [0.0, 0.4]
    torch.testing.assert_close(table.r, torch.tensor([1e-5, 1.5e-5, 2.25e-5], dtype=torch.float64))


def test_table_validation():
    r = torch.logspace(-3, 1, 8, dtype=torch.float64)
    with pytest.raises(ValueError):
        DipoleTable(r=r, y=torch.zeros(1, dtype=torch.float64), N=torch.zeros((2, 8), dtype=torch.float64), x0=0.01)
    with pytest.raises(ValueError):
        DipoleTable(r=r.flip(0), y=torch.zeros(1, dtype=torch.float64), N=torch.zeros((1, 8), dtype=torch.float64),
                    x0=0.01)


def test_initial_conditions(tmp_path):
    r = torch.logspace(-7, 2, 50, dtype=torch.float64)
    mv = MV(qs0sqr=0.2).dipole_amplitude(r)
    assert bool(((mv >= 0) & (mv <= 1)).all())
    head = bk_table_mc50w()["ic_head"]
    path = tmp_path / "ic.dat"
    np.savetxt(path, head)
    ic = ICDataFile(path, x0=0.01)
    torch.testing.assert_close(ic.dipole_amplitude(ic.r), ic.N, rtol=1e-12, atol=1e-30)
    assert ic.dipole_amplitude(torch.tensor([1e-12], dtype=torch.float64)).item() == 0.0
    assert ic.dipole_amplitude(torch.tensor([1e6], dtype=torch.float64)).item() == 1.0
    short = tmp_path / "short.dat"
    np.savetxt(short, head[:5])
    with pytest.raises(ValueError):
        ICDataFile(short)


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "nlo_b200.h").read_text()
    declared = set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(nlo_\w+)\(", header, flags=re.M))
    assert declared, "no declarations parsed"
    lib = ctypes.CDLL(str(_native.LIBRARY_PATH))
    missing = [name for name in sorted(declared) if not hasattr(lib, name)]
    assert not missing, missing
    assert set(_native.EXPORTED) <= declared


def test_library_rejects_bad_arguments_without_a_gpu():
    lib = _native.load()
    assert lib.nlo_abi_version() == 1
    dirs = _native.sobol_dirs(4, 0)
    # invalid precision and NULL buffers are rejected on the host before any launch
    assert lib.nlo_sobol_draw(dirs, 0, 16, 7, None, None) == 1
    assert lib.nlo_bk_splines(None, None, 2, 1, None, None) == 1
    assert b"spline" in lib.nlo_last_error()
    params = _native.BKParams()
    params.nc, params.nf, params.lambda_qcd, params.c2, params.ksub = 3.0, 4.0, 0.241, 1.0, 0.65
    assert lib.nlo_bk_k1(params, None, 10, None, None, None, None, None) == 1
    assert b"NF" in lib.nlo_last_error()
    assert lib.nlo_bk_k2kf_workspace_bytes(400) > 0
    assert lib.nlo_bk_spline_doubles(400) == 400 + 8 * 399 + 2 * 400
    # the multi-set evolution checks its sets, budgets, directions and waves on the host
    import ctypes

    params.nf = 3.0
    tables = (ctypes.c_void_p * 2)(16, 32)
    budgets = (ctypes.c_int64 * 2)(1024, 1 << 31)
    sets_dirs = (_native.SobolDirs * 2)(dirs, dirs)
    box = _native.box([0.0] * 4, [1.0] * 4)

    def sets_call(n, waves=4, tabs=tables, samples=budgets, d=sets_dirs):
        return lib.nlo_bk_evolve_sets(params, 64, 64, n, tabs, 1, 0.2, 2, d, samples, box, waves, 128, 256,
                                      1 << 30, None)

    assert sets_call(0) == 1 and b"sets" in lib.nlo_last_error()
    assert sets_call(300) == 1 and b"sets" in lib.nlo_last_error()
    assert sets_call(2, waves=0) == 1 and b"waves" in lib.nlo_last_error()
    assert sets_call(2) == 1 and b"samples" in lib.nlo_last_error()  # 2^31 > 2^30
    assert sets_call(1, tabs=(ctypes.c_void_p * 1)(None)) == 1 and b"table" in lib.nlo_last_error()
    bad = _native.sobol_dirs(4, 0)
    bad.dims = 2
    assert sets_call(1, d=(_native.SobolDirs * 1)(bad)) == 1 and b"set 0" in lib.nlo_last_error()
    assert lib.nlo_bk_sets_workspace_bytes(64, 257, 4) == 0
    assert lib.nlo_bk_sets_workspace_bytes(64, 2, 4) > 0


def test_c_struct_layouts_match_ctypes(tmp_path):
    """The ctypes mirrors of the C structs have the C header's sizes and offsets."""
    import ctypes
    import shutil
    import subprocess

    from nlo_bk_optimized_b200 import _native

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    root = Path(__file__).resolve().parents[1]
    src = tmp_path / "layout.c"
    src.write_text(
        "#include <stdio.h>\n#include <stddef.h>\n#include \"nlo_b200.h\"\n"
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(nlo_dis_kinematics),"
        " offsetof(nlo_dis_kinematics, maxr), offsetof(nlo_dis_kinematics, max_alpha), sizeof(nlo_dipole),"
        " offsetof(nlo_dipole, table), sizeof(nlo_vegas_options), offsetof(nlo_vegas_options, keep_edges),"
        " sizeof(nlo_bk_params), offsetof(nlo_bk_params, order), offsetof(nlo_bk_params, rc_nlo));return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-I", str(root / "include"), str(src), "-o", str(exe)], check=True)
    c = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    py = [ctypes.sizeof(_native.DisKinematics), _native.DisKinematics.maxr.offset,
          _native.DisKinematics.max_alpha.offset, ctypes.sizeof(_native.Dipole), _native.Dipole.table.offset,
          ctypes.sizeof(_native.VegasOptions), _native.VegasOptions.keep_edges.offset,
          ctypes.sizeof(_native.BKParams), _native.BKParams.order.offset, _native.BKParams.rc_nlo.offset]
    assert c == py


def test_serving_helpers():
    """Rapidity range and Vegas settings of a served request, and the latency quantiles."""
    import math

    from nlo_bk_optimized_b200.serving import ServerStats, dis_options_for, maxy_for

    assert maxy_for([(10.0, 1e-3)], step=0.2) >= math.log(10.0 / 1e-3)
    assert abs(maxy_for([(10.0, 1e-3)], step=0.2) / 0.2 - round(maxy_for([(10.0, 1e-3)], step=0.2) / 0.2)) < 1e-9
    assert dis_options_for(1 << 20)["vegas_samples"] == (1 << 20) // 16
    assert dis_options_for(1 << 10)["vegas_samples"] == 4096
    stats = ServerStats(latencies=[0.1 * k for k in range(1, 101)], points=300, requests=100, started=0.0,
                        finished=10.0)
    summary = stats.summary()
    assert summary["p50_s"] == pytest.approx(5.0)
    assert summary["p99_s"] == pytest.approx(9.9)
    assert summary["points_per_s"] == pytest.approx(30.0)


def test_dis_budget_split_and_seed_plan():
    """The Vegas budget split of _vegas_with_budget (dis/observables.py:667-692) and the seed
    offsets of sigma_dip_d2b / sigma_qg_d2b (dis/observables.py:387-532), planned on the host."""
    from nlo_bk_optimized_b200.dipole import GBW
    from nlo_bk_optimized_b200.dis import DISConfig, DISOrder, Polarization, Quark, QuarkType
    from nlo_bk_optimized_b200.dis.observables import TERMS, _Engine, _plan_sigma
    from nlo_bk_optimized_b200.numerics.integration import budget_options

    o = budget_options(2_000_000, 1e-3)
    assert (o.max_iterations, o.samples_per_iteration, o.min_iterations) == (8, 250_000, 3)
    o = budget_options(5, 1e-3)
    assert (o.max_iterations, o.samples_per_iteration, o.min_iterations) == (2, 2, 2)
    with pytest.raises(ValueError):
        budget_options(1, 1e-3)
    config = DISConfig(order=DISOrder.NLO, quarks=(Quark(QuarkType.LIGHT, 0.14), Quark(QuarkType.C, 1.4)),
                       maxeval=1000)
    engine = _Engine(GBW(), config, torch.device("cpu"))
    plan = _plan_sigma(engine, 10.0, 1e-3, Polarization.T, seed=7, points=24, overrides={})
    dip_seeds = [j.seed for jobs in plan.dip for j in jobs if j.options is not None]
    qg_seeds = [j.seed for jobs in plan.qg for j in jobs]
    assert dip_seeds == [7, 8, 9, 10]
    assert qg_seeds == [107, 108, 109, 110, 111, 112]
    # light quarks get 10x the virtual-term budget
    light, charm = plan.dip[0][1].options, plan.dip[1][1].options
    assert light.samples_per_iteration * light.max_iterations == 10_000
    assert charm.samples_per_iteration * charm.max_iterations == 1000
    assert [j.term for j in plan.qg[0]] == [TERMS["I1"], TERMS["I2N"], TERMS["I3N"]]
    assert plan.lo.kin.xbj == 1.0  # NLO: LO term at x_Bj = X0


def test_kinematical_constraint_entry_points_validate_on_the_host():
    """The constraint reads the amplitude history: the entry points without one refuse it,
    and the history evolution refuses steppers other than Euler, before anything launches."""
    import ctypes

    from nlo_bk_optimized_b200 import _native
    from nlo_bk_optimized_b200.bk.config import BKConfig
    from nlo_bk_optimized_b200.bk.evolution import params_of

    lib = _native.load()
    config = BKConfig(KINEMATICAL_CONSTRAINT=True, EULER_METHOD=True)
    params = params_of(config, _native.PRECISION_FP64)
    assert params.kinematical_constraint == 1
    dirs = _native.sobol_dirs(4, 0)
    box = _native.box([0.0] * 4, [1.0] * 4)
    fake = ctypes.c_void_p(16)  # never dereferenced: validation fails first
    rc = lib.nlo_bk_evolve(params, fake, 32, 1, 0.2, _native.STEPPERS["euler"], dirs, 16, box, fake, fake, fake,
                           1 << 30, None)
    assert rc == 1 and b"history" in lib.nlo_last_error()
    rc = lib.nlo_bk_rhs(params, fake, fake, 32, dirs, 16, box, fake, None, None, fake, 1 << 30, None)
    assert rc == 1 and b"history" in lib.nlo_last_error()
    rc = lib.nlo_bk_evolve_history(params, fake, 32, fake, 0, 1, 0.2, _native.STEPPERS["rk4"], dirs, 16, box, fake,
                                   fake, fake, 1 << 30, None)
    assert rc == 1 and b"Euler" in lib.nlo_last_error()


def test_fixed_step_evolutions_reject_the_adaptive_stepper():
    """The batched, sharded and served evolutions advance rows by fixed device steps."""
    import torch

    from nlo_bk_optimized_b200 import BKConfig
    from nlo_bk_optimized_b200.bk.batch import evolve_batch
    from nlo_bk_optimized_b200.bk.config import IntegrationMethod, require_fixed_step

    config = BKConfig(STEPPER="rk2_adaptive", INTMETHOD_NLO=IntegrationMethod.SOBOL)
    with pytest.raises(ValueError, match="rk2_adaptive"):
        evolve_batch(torch.zeros((1, 8), dtype=torch.float64), torch.ones(8, dtype=torch.float64), 1, config, [16])
    with pytest.raises(ValueError, match="fixed-step"):
        require_fixed_step(config, "the sharded evolution")
    require_fixed_step(BKConfig(STEPPER="rk4"), "the sharded evolution")
