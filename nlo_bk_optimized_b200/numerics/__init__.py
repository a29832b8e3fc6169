"""Host-side numerical helpers and the general Vegas integrator."""

from nlo_bk_optimized_b200.numerics.integration import IntegralResult, VegasState, vegas
from nlo_bk_optimized_b200.numerics.interpolation import MIN_LOG_VALUE, NaturalCubicSpline

__all__ = ["IntegralResult", "MIN_LOG_VALUE", "NaturalCubicSpline", "VegasState", "vegas"]
