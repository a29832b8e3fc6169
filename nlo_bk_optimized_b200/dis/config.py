"""DIS constants, quarks and switches: the public interface of the reference's
``dis/config.py`` (torch_nlo_clean/src/nlo_torch/dis/config.py:1-153), with the same
names, defaults and validation, so code written against it keeps working.

Two fields are added for the device integrator: ``vegas_bins`` (32, the reference's
``vegas`` default) and ``precision`` ("mixed": FP32 integrands with FP64 sums; "fp64").
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from enum import Enum, auto

LambdaQCD = 0.241
AlphaEM = 1 / 137.035999
NC = 3
CF = (NC**2 - 1) / (2 * NC)
Q0sqr = 1.0


class Polarization(Enum):
    T = auto()
    L = auto()


class DISOrder(Enum):
    LO = auto()
    NLO = auto()


class NcScheme(Enum):
    FiniteNC = auto()
    LargeNC = auto()


class RunningCouplingScheme(Enum):
    SMALLEST = auto()
    PARENT = auto()


class RunningCouplingIRScheme(Enum):
    FREEZE = auto()
    SMOOTH = auto()


class HeavyQuarkX(Enum):
    MassDependentX = auto()
    MassIndependentX = auto()


class QuarkType(Enum):
    U = auto()
    D = auto()
    S = auto()
    C = auto()
    B = auto()
    T = auto()
    LIGHT = auto()


_UNSET = object()
_DEFAULT_MASS = {
    QuarkType.U: 0.002, QuarkType.D: 0.002, QuarkType.S: 0.002, QuarkType.LIGHT: 0.002,
    QuarkType.C: 1.4, QuarkType.B: 4.18, QuarkType.T: 173.0,
}


@dataclass(frozen=True, slots=True, init=False)
class Quark:
    """A quark flavour and mass.  ``Quark()`` is a light quark of mass 1 MeV; a given
    type without a mass takes the reference's default for it (dis/config.py:56-87)."""

    type: QuarkType
    mass: float

    def __init__(self, type: QuarkType | object = _UNSET, mass: float | None = None) -> None:  # noqa: A002
        flavour = QuarkType.LIGHT if type is _UNSET else type
        if not isinstance(flavour, QuarkType):
            raise TypeError("type must be a QuarkType")
        if mass is None:
            mass = 0.001 if type is _UNSET else _DEFAULT_MASS[flavour]
        object.__setattr__(self, "type", flavour)
        object.__setattr__(self, "mass", float(mass))

    @property
    def charge(self) -> float:
        """Electric charge; LIGHT stands for u+d+s and carries sqrt(4/9 + 1/9 + 1/9)."""
        if self.type in (QuarkType.U, QuarkType.C):
            return 2 / 3
        if self.type in (QuarkType.D, QuarkType.S, QuarkType.B):
            return -1 / 3
        if self.type is QuarkType.LIGHT:
            return math.sqrt(2 / 3)
        raise ValueError("the source does not define an electric charge for the top quark")


@dataclass(frozen=True, slots=True)
class DISConfig:
    order: DISOrder = DISOrder.LO
    nc_scheme: NcScheme = NcScheme.FiniteNC
    rc_scheme: RunningCouplingScheme = RunningCouplingScheme.SMALLEST
    rc_ir_scheme: RunningCouplingIRScheme = RunningCouplingIRScheme.FREEZE
    maxr: float = 30.0
    C2_alpha: float = 1.0
    nf_alphas: int = -1
    max_alpha_s_freeze: float = 0.7
    heavy_quark_x_scheme: HeavyQuarkX = HeavyQuarkX.MassIndependentX
    transverse_area: float = 1.0
    maxeval: int = 2_000_000
    epsrel: float = 0.001
    cuda_fusion: bool = True
    cuda_nested: bool = True
    cuda_nested_points: int = 48
    quarks: tuple[Quark, ...] = field(default_factory=lambda: (Quark(QuarkType.LIGHT), Quark(QuarkType.C)))
    vegas_bins: int = 32
    precision: str = "mixed"

    def __post_init__(self) -> None:
        if self.maxr <= 0 or self.C2_alpha <= 0:
            raise ValueError("maxr and C2_alpha must be positive")
        if self.max_alpha_s_freeze <= 0 or self.transverse_area <= 0:
            raise ValueError("coupling freeze and transverse area must be positive")
        if self.maxeval < 1 or self.epsrel <= 0:
            raise ValueError("integration budget and relative accuracy must be positive")
        if not 8 <= self.cuda_nested_points <= 128:
            raise ValueError("nested DIS integration requires 8 to 128 inner points")
        if not self.quarks:
            raise ValueError("at least one quark is required")
        if len(self.quarks) > 8:
            raise ValueError("at most eight quarks are supported")
        if not 2 <= self.vegas_bins <= 256:
            raise ValueError("vegas_bins must lie in 2..256")
        if self.precision not in ("mixed", "fp64"):
            raise ValueError("precision must be 'mixed' or 'fp64'")

    @property
    def active_flavors(self) -> int:
        if self.nf_alphas >= 0:
            return self.nf_alphas
        return sum(3 if quark.type is QuarkType.LIGHT else 1 for quark in self.quarks)


__all__ = [
    "AlphaEM",
    "CF",
    "DISConfig",
    "DISOrder",
    "HeavyQuarkX",
    "LambdaQCD",
    "NC",
    "NcScheme",
    "Polarization",
    "Q0sqr",
    "Quark",
    "QuarkType",
    "RunningCouplingIRScheme",
    "RunningCouplingScheme",
]
