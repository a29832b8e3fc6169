"""Host-side numerical helpers."""

from nlo_bk_optimized_b200.numerics.interpolation import MIN_LOG_VALUE, NaturalCubicSpline

__all__ = ["MIN_LOG_VALUE", "NaturalCubicSpline"]
