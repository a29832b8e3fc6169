"""BK evolution configuration (mirrors torch_nlo_clean/src/nlo_torch/bk/config.py:1-134).

Field names, enum names, defaults and validation follow the reference ``BKConfig``
so that user code constructs it unchanged.  Additions for the B200 path:

* ``IntegrationMethod.VEGAS`` (the default, as in the reference) integrates K2+Kf per
  parent by Vegas on the device with the reference's settings (32 bins, warm-up
  max(2, MCINTPOINTS/5), 2..4 iterations of MCINTPOINTS, epsrel 0.2) and, with
  ``VEGAS_REUSE_GRID``, each parent's grid carried through the evolution with a warm-up
  shortened by ``VEGAS_REUSE_WARMUP_FRACTION``.  ``IntegrationMethod.SOBOL`` (new) is
  quasi-Monte Carlo on the first ``MCINTPOINTS`` points of ``SobolEngine(4,
  scramble=True, seed)`` for every parent and stage: the fast B200 path, which the
  headline benchmark uses.  MISER and MULTIPLE are accepted by the dataclass and rejected
  by the device path.
* ``STEPPER`` -- "rk3" (the default: the reference's Kutta RK3 of its CUDA production
  path, bk/evolution.py:190-236), "rk4" (classical), "euler", or "rk2_adaptive" (the
  reference's adaptive midpoint stepper with step doubling, its stepper off the CUDA float32
  path, bk/evolution.py:239-326, with DE_SOLVER_ABSERR / DE_SOLVER_RELERR; driven from the
  host, one error read per attempt; not for the batched, sharded or served evolutions);
  ``EULER_METHOD=True`` selects "euler".
* ``PRECISION`` -- "mixed" (FP32 integrands, FP64 sums/splines/RK update) or
  "fp64"; ``None`` picks "mixed" for float32 tables and "fp64" otherwise.
* ``ALPHA_S_CAP`` -- if positive, alpha_s = min(alpha_s, ALPHA_S_CAP)
  (the frozen-coupling variant).
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import Enum, auto


class RunningCouplingLO(Enum):
    FIXED_LO = auto()
    PARENT_LO = auto()
    SMALLEST_LO = auto()
    BALITSKY_LO = auto()
    FAC_LO = auto()
    BEUF_LO = auto()


class RunningCouplingNLO(Enum):
    FIXED_NLO = auto()
    PARENT_NLO = auto()
    SMALLEST_NLO = auto()


class ResummationCoupling(Enum):
    RESUM_RC_PARENT = auto()
    RESUM_RC_SMALLEST = auto()
    RESUM_RC_FIXED = auto()


class IntegrationMethod(Enum):
    VEGAS = auto()
    MISER = auto()
    MULTIPLE = auto()
    SOBOL = auto()


class BKOrder(Enum):
    LO = auto()
    LO_RESUM_DLOG = auto()
    LO_RESUM_DLOG_SLOG = auto()
    NLO = auto()
    NLO_RESUM_DLOG = auto()
    NLO_RESUM_DLOG_SLOG = auto()

    @property
    def has_nlo_kernels(self) -> bool:
        return self in {BKOrder.NLO, BKOrder.NLO_RESUM_DLOG, BKOrder.NLO_RESUM_DLOG_SLOG}

    @property
    def resum_dlog(self) -> bool:
        return self in {
            BKOrder.LO_RESUM_DLOG,
            BKOrder.LO_RESUM_DLOG_SLOG,
            BKOrder.NLO_RESUM_DLOG,
            BKOrder.NLO_RESUM_DLOG_SLOG,
        }

    @property
    def resum_slog(self) -> bool:
        return self in {BKOrder.LO_RESUM_DLOG_SLOG, BKOrder.NLO_RESUM_DLOG_SLOG}


STEPPERS = ("rk3", "rk4", "euler", "rk2_adaptive")
PRECISIONS = ("mixed", "fp64")


@dataclass(frozen=True, slots=True)
class BKConfig:
    NC: float = 3.0
    NF: int = 3
    LambdaQCD: float = 0.241
    RINTPOINTS: int = 85
    THETAINTPOINTS: int = 85
    INTACCURACY: float = 0.001
    MCINTACCURACY: float = 0.2
    MAXR: float = 30.0
    MINR: float = 1e-6
    RPOINTS: int = 100
    MCINTPOINTS: int = 100_000
    DE_SOLVER_STEP: float = 0.2
    DE_SOLVER_ABSERR: float = 1e-6
    DE_SOLVER_RELERR: float = 1e-4
    FIXED_AS: float = 0.2
    RC_LO: RunningCouplingLO = RunningCouplingLO.BALITSKY_LO
    RC_NLO: RunningCouplingNLO = RunningCouplingNLO.SMALLEST_NLO
    RESUM_RC: ResummationCoupling = ResummationCoupling.RESUM_RC_SMALLEST
    INTMETHOD_NLO: IntegrationMethod = IntegrationMethod.VEGAS
    FORCE_POSITIVE_N: bool = True
    SYMMETRIZE_Z_Z2_INTEGRATION: bool = True
    DNDY: bool = False
    Order: BKOrder = BKOrder.NLO_RESUM_DLOG_SLOG
    KSUB: float = 0.65
    KINEMATICAL_CONSTRAINT: bool = False
    EULER_METHOD: bool = False
    C2: float = 1.0
    CUDA_FUSION: bool = True
    K1_FIXED: bool = True
    K1_FIXED_REFINE: bool = False
    VEGAS_REUSE_GRID: bool = True
    VEGAS_REUSE_WARMUP_FRACTION: float = 0.25
    STEPPER: str = "rk3"
    PRECISION: str | None = None
    ALPHA_S_CAP: float = 0.0

    def __post_init__(self) -> None:
        # bk/config.py:103-124
        if self.NF not in {0, 3, 5}:
            raise ValueError("NF must be 0, 3, or 5")
        if self.MINR <= 0 or self.MAXR <= self.MINR or self.RPOINTS < 2:
            raise ValueError("the BK r grid requires 0 < MINR < MAXR and RPOINTS >= 2")
        if self.RINTPOINTS < 1 or self.THETAINTPOINTS < 1 or self.MCINTPOINTS < 1:
            raise ValueError("integration limits must be positive")
        if self.INTACCURACY <= 0 or self.MCINTACCURACY <= 0:
            raise ValueError("integration accuracies must be positive")
        if not 0 <= self.VEGAS_REUSE_WARMUP_FRACTION <= 1:
            raise ValueError("VEGAS_REUSE_WARMUP_FRACTION must lie between zero and one")
        if self.DE_SOLVER_STEP <= 0:
            raise ValueError("DE_SOLVER_STEP must be positive")
        if self.C2 <= 0 or self.KSUB <= 0:
            raise ValueError("C2 and KSUB must be positive")
        fixed_LO = self.RC_LO is RunningCouplingLO.FIXED_LO
        fixed_NLO = self.RC_NLO is RunningCouplingNLO.FIXED_NLO
        if fixed_LO != fixed_NLO:
            raise ValueError("fixed coupling must be selected for both RC_LO and RC_NLO")
        if self.KINEMATICAL_CONSTRAINT and not self.EULER_METHOD:
            raise ValueError("KINEMATICAL_CONSTRAINT requires EULER_METHOD")
        if self.STEPPER not in STEPPERS:
            raise ValueError(f"STEPPER must be one of {STEPPERS}")
        if self.PRECISION is not None and self.PRECISION not in PRECISIONS:
            raise ValueError(f"PRECISION must be None or one of {PRECISIONS}")
        if self.ALPHA_S_CAP < 0:
            raise ValueError("ALPHA_S_CAP must be non-negative")
        if self.MCINTPOINTS > 1 << 30:
            raise ValueError("MCINTPOINTS may not exceed 2^30 Sobol points")

    @property
    def stepper(self) -> str:
        return "euler" if self.EULER_METHOD else self.STEPPER


def device_supported(config: BKConfig) -> str | None:
    """Return why a configuration is outside the device kernels, or None.

    Every Order, RC_LO, RC_NLO, RESUM_RC and NF of BKConfig, and the kinematical
    constraint, run on the device; K2+Kf integrates by VEGAS or SOBOL."""

    if config.Order.has_nlo_kernels and config.INTMETHOD_NLO not in (IntegrationMethod.VEGAS,
                                                                     IntegrationMethod.SOBOL):
        return (f"the device K2+Kf integrates with IntegrationMethod.VEGAS or SOBOL, not "
                f"{config.INTMETHOD_NLO.name}")
    return None


def require_sobol(config: BKConfig, what: str) -> None:
    """The batched and served evolutions take a Monte Carlo budget per parameter set or
    request as a Sobol point count, so they integrate K2+Kf by IntegrationMethod.SOBOL."""
    if config.Order.has_nlo_kernels and config.INTMETHOD_NLO is not IntegrationMethod.SOBOL:
        raise ValueError(f"{what} integrates K2+Kf with IntegrationMethod.SOBOL (its budgets are Sobol point "
                         f"counts); got {config.INTMETHOD_NLO.name}")


def require_fixed_step(config: BKConfig, what: str) -> None:
    """The batched, sharded and served evolutions advance every row by fixed steps on the
    device; the adaptive stepper's accept/retry decisions are per evolution on the host."""
    if config.stepper == "rk2_adaptive":
        raise ValueError(f"{what} takes the fixed-step steppers (rk3, rk4, euler), not rk2_adaptive")


ORDER_CODES = {
    BKOrder.NLO_RESUM_DLOG_SLOG: 0,
    BKOrder.NLO_RESUM_DLOG: 1,
    BKOrder.NLO: 2,
    BKOrder.LO_RESUM_DLOG_SLOG: 3,
    BKOrder.LO_RESUM_DLOG: 4,
    BKOrder.LO: 5,
}
RC_LO_CODES = {
    RunningCouplingLO.BALITSKY_LO: 0,
    RunningCouplingLO.FIXED_LO: 0,  # the Balitsky form with a constant coupling
    RunningCouplingLO.PARENT_LO: 1,
    RunningCouplingLO.SMALLEST_LO: 2,
    RunningCouplingLO.FAC_LO: 3,
    RunningCouplingLO.BEUF_LO: 4,
}
RESUM_RC_CODES = {
    ResummationCoupling.RESUM_RC_SMALLEST: 0,
    ResummationCoupling.RESUM_RC_PARENT: 1,
    ResummationCoupling.RESUM_RC_FIXED: 2,
}
RC_NLO_CODES = {
    RunningCouplingNLO.SMALLEST_NLO: 0,
    RunningCouplingNLO.FIXED_NLO: 0,  # with the constant coupling
    RunningCouplingNLO.PARENT_NLO: 1,
}


def fixed_coupling(config: BKConfig) -> bool:
    """_alpha_s is the constant FIXED_AS when either coupling choice is fixed
    (bk_kernels/k1.py:158-170, bk/derivatives.py:775-787)."""
    return config.RC_LO is RunningCouplingLO.FIXED_LO or config.RC_NLO is RunningCouplingNLO.FIXED_NLO


__all__ = [
    "BKConfig",
    "BKOrder",
    "IntegrationMethod",
    "ResummationCoupling",
    "RunningCouplingLO",
    "RunningCouplingNLO",
    "device_supported",
    "fixed_coupling",
    "require_sobol",
]
