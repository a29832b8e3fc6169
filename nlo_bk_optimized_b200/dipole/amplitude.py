"""GBW and BK-table dipole amplitudes (interface of the reference's
dipole/amplitude.py:23-302), evaluated on the device by libnlo_b200.so.

``BKDipole`` keeps the table prepared for the device (nlo_dis_table_prepare_interpolated):
with the default SPLINE_LINEAR interpolation the local 7/9-point splines of every r
interval are precomputed once; LINEAR_LINEAR interpolates bilinearly in (r, Y)
(dipole/amplitude.py:188-212).
``initialize_interpolation(Y)`` fits the global spline at one rapidity on the device,
exactly as the reference's state machine does.  Evaluation needs CUDA tensors; there is
no CPU path.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from enum import Enum, auto

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.dipole.table import DipoleTable


class AmplitudeInterpolation(Enum):
    SPLINE_LINEAR = auto()
    LINEAR_LINEAR = auto()


@dataclass(frozen=True, slots=True)
class GBW:
    Qs0sqr: float = 0.1
    lambda_: float = 0.3
    gamma: float = 1.0
    x0: float = 1.0

    @property
    def min_r(self) -> float:
        return 1e-30

    @property
    def max_r(self) -> float:
        return 1e3

    def X0(self) -> float:
        return self.x0

    def native(self) -> _native.Dipole:
        d = _native.Dipole()
        d.kind = _native.DIPOLE_GBW
        d.qs0sqr, d.lambda_, d.gamma, d.x0 = self.Qs0sqr, self.lambda_, self.gamma, self.x0
        return d

    def dipole_amplitude(self, r: torch.Tensor, Y: torch.Tensor) -> torch.Tensor:
        return _evaluate(self.native(), r, Y)

    def saturation_scale(self, Y: torch.Tensor, Ns: float) -> torch.Tensor:
        return _saturation_scale(self, Y, Ns)


def _evaluate(dipole: _native.Dipole, r: torch.Tensor, Y: torch.Tensor) -> torch.Tensor:
    r, Y = torch.broadcast_tensors(torch.as_tensor(r), torch.as_tensor(Y, device=torch.as_tensor(r).device))
    _native.require_cuda(r.contiguous(), "r")
    shape, dtype = r.shape, r.dtype
    r64 = r.reshape(-1).to(torch.float64).contiguous()
    Y64 = Y.reshape(-1).to(device=r.device, dtype=torch.float64).contiguous()
    out = torch.empty_like(r64)
    precision = _native.PRECISION_FP64 if dtype == torch.float64 else _native.PRECISION_MIXED
    lib = _native.load()
    with torch.cuda.device(r.device):
        _native.check(lib.nlo_dis_dipole_amplitude(ctypes.byref(dipole), r64.data_ptr(), Y64.data_ptr(), r64.numel(),
                                                   precision, out.data_ptr(), _native.stream_handle(r.device)))
    return out.reshape(shape).to(dtype)


class BKDipole:
    """Dipole amplitude from a BK table (dipole/amplitude.py:48-252)."""

    def __init__(self, table: DipoleTable,
                 interpolation: AmplitudeInterpolation = AmplitudeInterpolation.SPLINE_LINEAR) -> None:
        if table.r.numel() < 9:
            raise ValueError("BKDipole requires at least nine r points")
        ratio = table.r[1] / table.r[0]
        expected = table.r[0] * torch.pow(ratio, torch.arange(table.r.numel(), dtype=table.r.dtype,
                                                              device=table.r.device))
        if not bool((torch.abs(expected / table.r - 1) <= 0.01).all()):
            raise ValueError("BKDipole requires a logarithmic r grid")
        if not isinstance(interpolation, AmplitudeInterpolation):
            raise TypeError("interpolation must be an AmplitudeInterpolation")
        self.table = table
        self.interpolation = interpolation
        Y0 = max(0.0, math.log(1 / table.x0))
        self.Y = table.y + Y0
        device = table.r.device if table.r.is_cuda else torch.device("cuda", torch.cuda.current_device())
        self.device = device
        nr, ny = table.r.numel(), table.y.numel()
        lib = _native.load()
        self._buffer = torch.empty(int(lib.nlo_dis_table_doubles(nr, ny)), dtype=torch.float64, device=device)
        r = table.r.to(device=device, dtype=torch.float64).contiguous()
        y = table.y.to(device=device, dtype=torch.float64).contiguous()
        N = table.N.to(device=device, dtype=torch.float64).contiguous()
        with torch.cuda.device(device):
            mode = 1 if interpolation is AmplitudeInterpolation.LINEAR_LINEAR else 0
            _native.check(lib.nlo_dis_table_prepare_interpolated(r.data_ptr(), y.data_ptr(), N.data_ptr(), nr, ny,
                                                                 float(table.x0), mode, self._buffer.data_ptr(),
                                                                 _native.stream_handle(device)))
        self._nr, self._ny = nr, ny
        self._min_Y = float(self.Y[0])
        self._max_Y = float(self.Y[-1])
        self._interpolator_Y = -1.0
        self._maxr_interpolate = -1.0

    @property
    def min_r(self) -> float:
        return float(self.table.r[0])

    @property
    def max_r(self) -> float:
        return float(self.table.r[-1])

    @property
    def min_Y(self) -> float:
        return self._min_Y

    @property
    def max_Y(self) -> float:
        return self._max_Y

    @property
    def maxr_interpolate(self) -> float:
        return self._maxr_interpolate

    def X0(self) -> float:
        return 1.0

    def native(self) -> _native.Dipole:
        d = _native.Dipole()
        d.kind = _native.DIPOLE_TABLE
        d.table = self._buffer.data_ptr()
        d.nr, d.ny = self._nr, self._ny
        return d

    def _matches(self, Y: float) -> bool:
        if abs(Y) < 0.001 and abs(self._interpolator_Y) < 0.001:
            return True
        den = min(Y, self._interpolator_Y)
        den = den if den != 0 else 1.0
        return self._interpolator_Y >= 0 and abs(Y - self._interpolator_Y) / den < 0.001

    def interpolator_initialized(self, Y: torch.Tensor) -> torch.Tensor:
        Yt = torch.as_tensor(Y, dtype=torch.float64)
        near_zero = (torch.abs(Yt) < 0.001) & (abs(self._interpolator_Y) < 0.001)
        den = torch.minimum(Yt, Yt.new_tensor(self._interpolator_Y))
        safe = torch.where(den != 0, den, torch.ones_like(Yt))
        match = (self._interpolator_Y >= 0) & (torch.abs(Yt - self._interpolator_Y) / safe < 0.001)
        return near_zero | match

    def initialize_interpolation(self, Y: float | torch.Tensor) -> None:
        value = float(Y.item()) if isinstance(Y, torch.Tensor) else float(Y)
        if 0 <= value <= self.min_Y:
            value = self.min_Y
        if value < 0:
            raise ValueError(f"cannot initialize interpolation at negative Y={value}")
        if value > self.max_Y:
            raise ValueError(f"cannot initialize interpolation at Y={value}; maximum is {self.max_Y}")
        if self._interpolator_Y >= 0 and self._matches(value):
            return
        lib = _native.load()
        with torch.cuda.device(self.device):
            _native.check(lib.nlo_dis_table_initialize(self._buffer.data_ptr(), self._nr, self._ny, value,
                                                       _native.stream_handle(self.device)))
        self._interpolator_Y = value
        self._maxr_interpolate = float(self._buffer[4])  # header slot written by the device search

    def check_rapidity(self, Y_max: float) -> None:
        """The reference raises ValueError when an evaluation reaches beyond the table."""
        if Y_max > self.max_Y:
            raise ValueError(f"Y must lie in [{self.min_Y}, {self.max_Y}] after initial-rapidity freezing")

    def dipole_amplitude(self, r: torch.Tensor, Y: torch.Tensor) -> torch.Tensor:
        Yt = torch.as_tensor(Y)
        if Yt.numel() and (float(Yt.max()) > self.max_Y or bool(((Yt < 0) & (Yt < self.min_Y)).any())):
            raise ValueError(f"Y must lie in [{self.min_Y}, {self.max_Y}] after initial-rapidity freezing")
        return _evaluate(self.native(), r, Y)

    def saturation_scale(self, Y: torch.Tensor, Ns: float) -> torch.Tensor:
        return _saturation_scale(self, Y, Ns)


def _saturation_scale(dipole: GBW | BKDipole, Y: torch.Tensor, Ns: float) -> torch.Tensor:
    """Bisection for N(r_s, Y) = Ns, returning 2/r_s^2 (dipole/amplitude.py:275-299)."""
    if Y.numel() != 1:
        raise ValueError("saturation_scale requires a scalar Y")
    device = Y.device if Y.is_cuda else torch.device("cuda", torch.cuda.current_device())
    Yd = Y.to(device=device, dtype=torch.float64).reshape(1)
    lower = torch.tensor([dipole.min_r * 1.0001], dtype=torch.float64, device=device)
    upper = torch.tensor([dipole.max_r * 0.999], dtype=torch.float64, device=device)
    lower_value = float(dipole.dipole_amplitude(lower, Yd)) - Ns
    upper_value = float(dipole.dipole_amplitude(upper, Yd)) - Ns
    if lower_value * upper_value > 0:
        raise ValueError("the saturation-scale bracket does not contain a root")
    lo, hi = float(lower), float(upper)
    for iteration in range(1, 1001):
        root = (lo + hi) / 2
        value = float(dipole.dipole_amplitude(torch.tensor([root], dtype=torch.float64, device=device), Yd)) - Ns
        if lower_value * value <= 0:
            hi = root
        else:
            lo = root
            lower_value = value
        if abs(hi - lo) < 1e-5 * min(abs(lo), abs(hi)) and iteration < 1000:
            return Y.new_tensor(2 / root**2)
    raise RuntimeError(f"saturation-scale root finding failed at Y={float(Y)}")


__all__ = ["AmplitudeInterpolation", "BKDipole", "GBW"]
