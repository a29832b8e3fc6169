"""``nlo-bk``: evolve a dipole amplitude with the BK equation on the device.

The options, their defaults and the output are those of the reference's command line
(cli/nlobk.py:21-148): ``--dndy`` prints "# r dN/dy[K1] dN/dy[K2+Kf] N" and one row per
active parent; otherwise the evolved table is written with ``save_bk_table`` in the
legacy text format and one summary line is printed.

Differences, all forced by the device path:

* ``--device`` defaults to ``cuda`` (the reference defaults to ``mps``); a non-CUDA
  device is an argument error.
* ``--integration`` adds ``sobol``, the fast quasi-Monte Carlo K2+Kf of the device; the
  default stays the reference's ``vegas``; ``miser``/``multiple`` are accepted and
  rejected like every other switch the device kernels do not implement, as an argument
  error naming it.
"""

from __future__ import annotations

import argparse
import sys

import torch

from nlo_bk_optimized_b200.bk.config import (
    BKConfig,
    BKOrder,
    IntegrationMethod,
    ResummationCoupling,
    RunningCouplingLO,
    RunningCouplingNLO,
    device_supported,
)
from nlo_bk_optimized_b200.bk.evolution import compute_dndy, solve_bk
from nlo_bk_optimized_b200.bk.initial_conditions import MV, ICDataFile
from nlo_bk_optimized_b200.dipole.table import save_bk_table

_ORDER = {
    "lo": BKOrder.LO,
    "lo_resum_dlog": BKOrder.LO_RESUM_DLOG,
    "lo_resum_dlog_slog": BKOrder.LO_RESUM_DLOG_SLOG,
    "nlo": BKOrder.NLO,
    "nlo_resum_dlog": BKOrder.NLO_RESUM_DLOG,
    "nlo_resum_dlog_slog": BKOrder.NLO_RESUM_DLOG_SLOG,
}
_RC_LO = {
    "fixed": RunningCouplingLO.FIXED_LO,
    "parent": RunningCouplingLO.PARENT_LO,
    "smallest": RunningCouplingLO.SMALLEST_LO,
    "balitsky": RunningCouplingLO.BALITSKY_LO,
    "fac": RunningCouplingLO.FAC_LO,
    "beuf": RunningCouplingLO.BEUF_LO,
}
_RC_NLO = {"parent": RunningCouplingNLO.PARENT_NLO, "smallest": RunningCouplingNLO.SMALLEST_NLO}
_RESUM_RC = {
    "parent": ResummationCoupling.RESUM_RC_PARENT,
    "smallest": ResummationCoupling.RESUM_RC_SMALLEST,
    "fixed": ResummationCoupling.RESUM_RC_FIXED,
}
_INTEGRATION = {
    "sobol": IntegrationMethod.SOBOL,
    "vegas": IntegrationMethod.VEGAS,
    "miser": IntegrationMethod.MISER,
    "multiple": IntegrationMethod.MULTIPLE,
}


def _parser() -> argparse.ArgumentParser:
    parser = argparse.ArgumentParser(prog="nlo-bk", description="Evolve a dipole amplitude with the BK equation")
    parser.add_argument("--ic-data", help="two-column r N initial condition")
    parser.add_argument("--x0", type=float, default=0.01)
    parser.add_argument("--qs0sqr", type=float, default=0.10)
    parser.add_argument("--gamma", type=float, default=1.0)
    parser.add_argument("--ec", type=float, default=1.0)
    parser.add_argument("--lambdaqcd", type=float, default=0.241)
    parser.add_argument("--maxy", type=float, default=10.0)
    parser.add_argument("--output", default="output.dat")
    parser.add_argument("--order", choices=tuple(_ORDER), default="nlo_resum_dlog_slog")
    parser.add_argument("--rc-lo", choices=tuple(_RC_LO), default="balitsky")
    parser.add_argument("--rc-nlo", choices=tuple(_RC_NLO), default="smallest")
    parser.add_argument("--resum-rc", choices=tuple(_RESUM_RC), default="smallest")
    parser.add_argument("--integration", choices=tuple(_INTEGRATION), default="vegas")
    parser.add_argument("--nf", type=int, choices=(0, 3, 5), default=3)
    parser.add_argument("--C2", type=float, default=1.0)
    parser.add_argument("--fixed-alpha-s", type=float, default=0.2)
    parser.add_argument("--Ksub", type=float, default=0.65)
    parser.add_argument("--minr", type=float, default=1e-6)
    parser.add_argument("--maxr", type=float, default=30.0)
    parser.add_argument("--rpoints", type=int, default=100)
    parser.add_argument("--mcintpoints", type=int, default=100_000)
    parser.add_argument("--step", type=float, default=0.2)
    parser.add_argument("--euler", action="store_true")
    parser.add_argument("--kinematical-constraint", action="store_true")
    parser.add_argument("--nolimit", action="store_true")
    parser.add_argument("--dndy", action="store_true")
    parser.add_argument("--seed", type=int)
    parser.add_argument("--device", default="cuda")
    parser.add_argument("--dtype", choices=("float32", "float64"), default="float32")
    return parser


def config_from_args(args: argparse.Namespace) -> BKConfig:
    """The BKConfig the reference's command line builds (cli/nlobk.py:41-60): a fixed LO
    coupling fixes the NLO coupling too."""
    fixed = args.rc_lo == "fixed"
    return BKConfig(
        NF=args.nf,
        MAXR=args.maxr,
        MINR=args.minr,
        RPOINTS=args.rpoints,
        MCINTPOINTS=args.mcintpoints,
        DE_SOLVER_STEP=args.step,
        FIXED_AS=args.fixed_alpha_s,
        RC_LO=_RC_LO[args.rc_lo],
        RC_NLO=RunningCouplingNLO.FIXED_NLO if fixed else _RC_NLO[args.rc_nlo],
        RESUM_RC=_RESUM_RC[args.resum_rc],
        INTMETHOD_NLO=_INTEGRATION[args.integration],
        FORCE_POSITIVE_N=not args.nolimit,
        DNDY=args.dndy,
        Order=_ORDER[args.order],
        KSUB=args.Ksub,
        KINEMATICAL_CONSTRAINT=args.kinematical_constraint,
        EULER_METHOD=args.euler,
        C2=args.C2,
    )


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
    why = device_supported(config)
    if why is not None:
        parser.error(f"not available on the device path: {why}")

    initial_condition = (
        ICDataFile(args.ic_data, x0=args.x0, device=device, dtype=dtype)
        if args.ic_data
        else MV(qs0sqr=args.qs0sqr, x0=args.x0, ec=args.ec, lambdaqcd=args.lambdaqcd, gamma=args.gamma)
    )

    if args.dndy:
        result = compute_dndy(initial_condition, config, device=device, dtype=dtype, seed=args.seed)
        print("# r dN/dy[K1] dN/dy[K2+Kf] N")
        rows = torch.stack((result.r, result.K1, result.K2_Kf, result.N), dim=1)
        for row in rows.detach().cpu().tolist():
            print(" ".join(f"{value:.15e}" for value in row))
        return 0

    table = solve_bk(initial_condition, args.maxy, config, device=device, dtype=dtype, seed=args.seed)
    save_bk_table(args.output, table)
    print(f"saved {table.y.numel()} rapidity slices and {table.r.numel()} r points to {args.output}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
