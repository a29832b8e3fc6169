"""Host-side cubic interpolation (numerics/interpolation.py:10-121 of the reference).

Used for preprocessing only (initial-condition files, table inspection); the
evolution refits its splines on the device (csrc/spline.cu).
"""

from __future__ import annotations

import torch

MIN_LOG_VALUE = -40.0


class NaturalCubicSpline:
    """Natural cubic spline whose knots occupy the last axis; coefficients a, b, c, d
    per interval, evaluated as a + dx (b + dx (c + dx d)) in the interval
    searchsorted(x, value, right=True) - 1 clamped to [0, n-2]."""

    def __init__(self, x: torch.Tensor, y: torch.Tensor) -> None:
        if x.ndim < 1 or y.ndim < 1:
            raise ValueError("x and y must have at least one dimension")
        if x.shape != y.shape:
            raise ValueError("x and y must have equal shapes")
        if x.shape[-1] < 3:
            raise ValueError("a cubic spline requires at least three points")
        if x.device != y.device or x.dtype != y.dtype:
            raise ValueError("x and y must have the same device and dtype")
        if not x.is_floating_point():
            raise TypeError("x and y must be floating-point tensors")
        if not bool(torch.isfinite(x).all()) or not bool(torch.isfinite(y).all()):
            raise ValueError("x and y must contain only finite values")
        h = x[..., 1:] - x[..., :-1]
        if not bool((h > 0).all()):
            raise ValueError("x must be strictly increasing")
        second = _second_derivatives(h, y)
        self.x = x
        self.a = y[..., :-1]
        self.b = (y[..., 1:] - y[..., :-1]) / h - h * (2 * second[..., :-1] + second[..., 1:]) / 6
        self.c = second[..., :-1] / 2
        self.d = (second[..., 1:] - second[..., :-1]) / (6 * h)

    def __call__(self, x: torch.Tensor) -> torch.Tensor:
        if self.x.ndim != 1:
            raise ValueError("evaluation is implemented for one-dimensional knot vectors")
        interval = (torch.searchsorted(self.x, x.contiguous(), right=True) - 1).clamp(0, self.x.shape[-1] - 2)
        dx = x - self.x[interval]
        return self.a[interval] + dx * (self.b[interval] + dx * (self.c[interval] + dx * self.d[interval]))


def _second_derivatives(h: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    """Interior second derivatives of the natural spline by the Thomas algorithm."""

    diagonal = 2 * (h[..., :-1] + h[..., 1:])
    off = h[..., 1:-1]
    rhs = 6 * ((y[..., 2:] - y[..., 1:-1]) / h[..., 1:] - (y[..., 1:-1] - y[..., :-2]) / h[..., :-1])
    m = diagonal.shape[-1]
    upper = torch.empty_like(diagonal)
    solution = torch.empty_like(diagonal)
    upper[..., 0] = off[..., 0] / diagonal[..., 0] if m > 1 else 0
    solution[..., 0] = rhs[..., 0] / diagonal[..., 0]
    for i in range(1, m):
        denominator = diagonal[..., i] - off[..., i - 1] * upper[..., i - 1]
        if i < m - 1:
            upper[..., i] = off[..., i] / denominator
        solution[..., i] = (rhs[..., i] - off[..., i - 1] * solution[..., i - 1]) / denominator
    for i in range(m - 2, -1, -1):
        solution[..., i] = solution[..., i] - upper[..., i] * solution[..., i + 1]
    zero = y.new_zeros((*y.shape[:-1], 1))
    return torch.cat((zero, solution, zero), dim=-1)


__all__ = ["MIN_LOG_VALUE", "NaturalCubicSpline"]
