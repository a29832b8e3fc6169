"""``nlo-dis``: DIS structure-function grids from a BK table on the device.

The options, defaults, run modes and output lines are those of the reference's command
line (cli/nlodis.py:46-163): the table is read with ``load_bk_table`` and interpolated
LINEAR_LINEAR, ``HERA_FL`` prints F_L at the twenty HERA (Q^2, x) points, ``F2FL_GRID``
prints F_2 and F_L of the light and charm quarks and the LO F_2 on the grid
Q^2 in {4.5, 45, 100}, x = 1e-5 * 1.5^k <= 1e-2; every integral reports its seed,
evaluation count, error and convergence on stderr.

The reference integrates point after point.  Here all points of a run mode go into one
batched device run per quark configuration (``structure_function_batch``); each value is
the one that point's ``FT``/``FL`` call gives when run alone with the same seed.

``--device`` defaults to ``cuda`` (the reference defaults to ``mps``); ``--dtype float64``
selects the all-FP64 integrands, ``float32`` the mixed build.
"""

from __future__ import annotations

import argparse
import sys
from dataclasses import replace

import torch

from nlo_bk_optimized_b200.dipole.amplitude import AmplitudeInterpolation, BKDipole
from nlo_bk_optimized_b200.dipole.table import load_bk_table
from nlo_bk_optimized_b200.dis.config import (
    DISConfig,
    DISOrder,
    Polarization,
    Quark,
    QuarkType,
    RunningCouplingIRScheme,
    RunningCouplingScheme,
)
from nlo_bk_optimized_b200.dis.observables import structure_function_batch
from nlo_bk_optimized_b200.numerics.integration import IntegralResult

# (Q^2 [GeV^2], x_Bj) of the HERA F_L points the reference prints (cli/nlodis.py:23-44)
HERA_FL_POINTS = (
    (1.5, 0.000028), (2.0, 0.000043), (2.5, 0.000059), (3.5, 0.000088), (5.0, 0.000129),
    (6.5, 0.000169), (8.5, 0.000224), (12.0, 0.000319), (15.0, 0.000402), (20.0, 0.000540),
    (25.0, 0.000687), (35.0, 0.000958), (45.0, 0.001210), (60.0, 0.001570), (90.0, 0.002430),
    (120.0, 0.003030), (150.0, 0.004020), (200.0, 0.005410), (250.0, 0.007360), (346.0, 0.009860),
)

# mb -> GeV^-2 factor the reference applies to --proton-area (cli/nlodis.py:67)
MB_TO_GEV2 = 2.56819


def grid_points() -> list[tuple[float, float]]:
    """(Q^2, x) of F2FL_GRID in the reference's order (cli/nlodis.py:98-103)."""
    points = []
    for Q2 in (4.5, 45.0, 100.0):
        x = 1e-5
        while x <= 1e-2:
            points.append((Q2, x))
            x *= 1.5
    return points


def _parser() -> argparse.ArgumentParser:
    parser = argparse.ArgumentParser(prog="nlo-dis", description="Calculate DIS structure-function grids")
    parser.add_argument("--name", default="nlodis")
    parser.add_argument("--datafile", required=True)
    parser.add_argument("--C2", type=float, required=True)
    parser.add_argument("--charm-mass", type=float, required=True)
    parser.add_argument("--light-mass", type=float, default=0.01)
    parser.add_argument("--proton-area", type=float, required=True, help="sigma_0/2 in mb")
    parser.add_argument("--rc-scheme", choices=("PARENT", "SMALLEST"), required=True)
    parser.add_argument("--order", choices=("LO", "NLO"), default="NLO")
    parser.add_argument("--runmode", choices=("F2FL_GRID", "HERA_FL"), default="HERA_FL")
    parser.add_argument("--epsrel", type=float, default=0.01)
    parser.add_argument("--mcintpoints", type=int, default=1_000_000)
    parser.add_argument("--nf", type=int, default=-1)
    parser.add_argument("--maxr", type=float, default=30.0)
    parser.add_argument("--quadrature-points", type=int, default=24)
    parser.add_argument("--batch-size", type=int, default=65_536)
    parser.add_argument("--seed", type=int, default=0)
    parser.add_argument("--device", default="cuda")
    parser.add_argument("--dtype", choices=("float32", "float64"), default="float32")
    parser.add_argument("--cuda-nested-points", type=int, default=48)
    parser.add_argument("--no-header", action="store_true")
    return parser


def config_from_args(args: argparse.Namespace) -> DISConfig:
    """The DISConfig of cli/nlodis.py:58-73 (light and charm quark, smooth IR coupling)."""
    return DISConfig(
        order=DISOrder[args.order],
        rc_scheme=RunningCouplingScheme[args.rc_scheme],
        rc_ir_scheme=RunningCouplingIRScheme.SMOOTH,
        maxr=args.maxr,
        C2_alpha=args.C2,
        nf_alphas=args.nf,
        transverse_area=args.proton_area * MB_TO_GEV2,
        maxeval=args.mcintpoints,
        epsrel=args.epsrel,
        cuda_nested_points=args.cuda_nested_points,
        quarks=(Quark(QuarkType.LIGHT, args.light_mass), Quark(QuarkType.C, args.charm_mass)),
        precision="fp64" if args.dtype == "float64" else "mixed",
    )


def _report(contribution: str, Q2: float, xbj: float, result: IntegralResult) -> None:
    print(f"# {contribution} Q2={Q2:.15g} x={xbj:.15g} seed={result.seed} n_eval={result.n_eval} "
          f"stderr={float(result.error):.8e} converged={result.converged}", file=sys.stderr)


def run_hera_fl(name: str, dipole: BKDipole, config: DISConfig, options: dict, single: bool) -> list[str]:
    seed = options["seed"]
    results = structure_function_batch([(Q2, x, Polarization.L, seed) for Q2, x in HERA_FL_POINTS], dipole, config,
                                       quadrature_points=options["quadrature_points"], single_precision=single)
    lines = []
    for (Q2, x), result in zip(HERA_FL_POINTS, results):
        lines.append(f"{name},{x:.15g},{Q2:.15g},{float(result.value):.15e}")
        _report("FL", Q2, x, result)
    return lines


def run_f2fl_grid(name: str, dipole: BKDipole, config: DISConfig, options: dict, single: bool) -> list[str]:
    seed, quad = options["seed"], options["quadrature_points"]
    points = grid_points()
    both = [(Q2, x, pol, seed) for Q2, x in points for pol in (Polarization.T, Polarization.L)]
    light, charm = config.quarks
    per_quark = {}
    for label, quark in (("light", light), ("charm", charm)):
        res = structure_function_batch(both, dipole, replace(config, quarks=(quark,)), quadrature_points=quad,
                                       single_precision=single)
        per_quark[label] = (res[0::2], res[1::2])
    # LO F_2 = F_T + F_L with F2's seed rule (F_L: seed + 1000)
    lo_points = [(Q2, x, pol, seed + (1000 if pol is Polarization.L else 0)) for Q2, x in points
                 for pol in (Polarization.T, Polarization.L)]
    lo = structure_function_batch(lo_points, dipole, replace(config, order=DISOrder.LO, quarks=(light, charm)),
                                  quadrature_points=quad, single_precision=single)
    lines = []
    for i, (Q2, x) in enumerate(points):
        FT_l, FL_l = per_quark["light"][0][i], per_quark["light"][1][i]
        FT_c, FL_c = per_quark["charm"][0][i], per_quark["charm"][1][i]
        F2_l = float(FT_l.value + FL_l.value)
        F2_c = float(FT_c.value + FL_c.value)
        F2_lo = float(lo[2 * i].value + lo[2 * i + 1].value)
        lines.append(f"{name},{x:.15g},{Q2:.15g},{F2_l:.15e},{float(FL_l.value):.15e},"
                     f"{F2_c:.15e},{float(FL_c.value):.15e},{F2_lo:.15e}")
        _report("FT_light", Q2, x, FT_l)
        _report("FL_light", Q2, x, FL_l)
        _report("FT_charm", Q2, x, FT_c)
        _report("FL_charm", Q2, x, FL_c)
    return lines


def main(argv: list[str] | None = None) -> int:
    parser = _parser()
    args = parser.parse_args(argv)
    device = torch.device(args.device)
    if device.type != "cuda":
        parser.error("the device path runs on CUDA devices; pass --device cuda")
    if not torch.cuda.is_available():
        parser.error("no CUDA device is available")
    dtype = torch.float32 if args.dtype == "float32" else torch.float64
    try:
        config = config_from_args(args)
    except ValueError as error:
        parser.error(str(error))
    table = load_bk_table(args.datafile, dtype=torch.float64, device=device)
    dipole = BKDipole(table, interpolation=AmplitudeInterpolation.LINEAR_LINEAR)
    options = {"quadrature_points": args.quadrature_points, "batch_size": args.batch_size, "seed": args.seed}
    single = dtype == torch.float32
    if args.runmode == "F2FL_GRID":
        if not args.no_header:
            print("fit,x,Q2,F2 light,FL light,F2 charm,FL charm,F2_LO")
        lines = run_f2fl_grid(args.name, dipole, config, options, single)
    else:
        if not args.no_header:
            print("fit,x,Q2,FL")
        lines = run_hera_fl(args.name, dipole, config, options, single)
    for line in lines:
        print(line)
    return 0


if __name__ == "__main__":
    sys.exit(main())
