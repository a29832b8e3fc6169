"""Initial conditions (mirrors torch_nlo_clean/src/nlo_torch/bk/initial_conditions.py:13-91).

They are evaluated once before the evolution; the evolution kernels only see the
resulting amplitude row.  A tabulated initial condition (``ICDataFile``) is fitted and
evaluated on the device (nlo_ic_spline / nlo_ic_evaluate) for CUDA tensors, which is the
path solve_bk and compute_dndy take; CPU tensors get the same spline on the host, as the
reference's own API allows.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from nlo_bk_optimized_b200.numerics.interpolation import NaturalCubicSpline


@dataclass(frozen=True, slots=True)
class MV:
    """McLerran-Venugopalan amplitude, initial_conditions.py:29-35:
    N = 1 - exp(-(r^2 Qs0^2)^gamma / 4 * log(1/(r Lambda) + ec e))."""

    qs0sqr: float = 0.10
    x0: float = 0.01
    ec: float = 1.0
    lambdaqcd: float = 0.241
    gamma: float = 1.0

    @property
    def min_r(self) -> float:
        return 1e-99

    @property
    def max_r(self) -> float:
        return 1e99

    def dipole_amplitude(self, r: torch.Tensor) -> torch.Tensor:
        exponent = (
            torch.pow(r.square() * self.qs0sqr, self.gamma)
            / 4
            * torch.log(1 / (r * self.lambdaqcd) + self.ec * 2.7182818)
        )
        return torch.where(exponent < 1e-5, exponent, 1 - torch.exp(-exponent))


def _read_table(path: Path) -> tuple[torch.Tensor, torch.Tensor]:
    """The (r, N) columns of a whitespace-separated text table in float64.  ``#`` starts a
    comment; blank lines are skipped; further columns are ignored."""
    try:
        data = np.loadtxt(path, comments="#", usecols=(0, 1), ndmin=2, dtype=np.float64)
    except ValueError as error:
        raise ValueError(f"{path}: every data line needs numeric r and N columns ({error})") from None
    r, N = torch.from_numpy(data[:, 0].copy()), torch.from_numpy(data[:, 1].copy())
    if r.numel() < 10:
        raise ValueError(f"{path}: {r.numel()} rows; a tabulated initial condition needs at least 10")
    if not (bool(torch.isfinite(r).all()) and bool(torch.isfinite(N).all())):
        raise ValueError(f"{path}: r and N must be finite")
    if not bool((r.diff() > 0).all()):
        raise ValueError(f"{path}: r must increase strictly from row to row")
    return r, N


class ICDataFile:
    """Tabulated initial condition (the reference's ICDataFile, bk/initial_conditions.py:38-91):
    a natural cubic spline through the rows of a two-column ``r N`` text file, with N = 0
    below its first r and N = 1 above its last."""

    def __init__(
        self,
        path: str | Path,
        *,
        x0: float = 0.01,
        dtype: torch.dtype = torch.float64,
        device: torch.device | str | None = None,
    ) -> None:
        self.path = Path(path)
        self.x0 = x0
        self._r64, self._N64 = _read_table(self.path)  # the file's values, the device fit's input
        self.r = self._r64.to(dtype=dtype, device=device)
        self.N = self._N64.to(dtype=dtype, device=device)
        self._host_spline: NaturalCubicSpline | None = None
        self._device_splines: dict[int, torch.Tensor] = {}

    @property
    def min_r(self) -> float:
        return float(self.r[0].item())

    @property
    def max_r(self) -> float:
        return float(self.r[-1].item())

    def device_spline(self, device: torch.device | str) -> torch.Tensor:
        """The spline buffer fitted on a CUDA device (nlo_ic_spline), cached per device."""
        from nlo_bk_optimized_b200 import _native

        device = torch.device(device)
        index = device.index if device.index is not None else torch.cuda.current_device()
        buffer = self._device_splines.get(index)
        if buffer is None:
            lib = _native.load()
            n = self._r64.numel()
            dev = torch.device("cuda", index)
            r = self._r64.to(dev)
            N = self._N64.to(dev)
            buffer = torch.empty(int(lib.nlo_ic_spline_doubles(n)), dtype=torch.float64, device=dev)
            with torch.cuda.device(dev):
                _native.check(lib.nlo_ic_spline(r.data_ptr(), N.data_ptr(), n, buffer.data_ptr(),
                                                _native.stream_handle(dev)))
            self._device_splines[index] = buffer
        return buffer

    def device_amplitude(self, r: torch.Tensor) -> torch.Tensor:
        """N at CUDA points r, in float64 (nlo_ic_evaluate)."""
        from nlo_bk_optimized_b200 import _native

        r = r.contiguous()
        _native.require_cuda(r, "r")
        spline = self.device_spline(r.device)
        r64 = r.to(torch.float64).contiguous()
        out = torch.empty_like(r64)
        lib = _native.load()
        with torch.cuda.device(r.device):
            _native.check(lib.nlo_ic_evaluate(spline.data_ptr(), self._r64.numel(), r64.data_ptr(), r64.numel(),
                                              out.data_ptr(), _native.stream_handle(r.device)))
        return out

    def dipole_amplitude(self, r: torch.Tensor) -> torch.Tensor:
        if r.is_cuda:
            return self.device_amplitude(r).to(self.r.dtype)
        if self._host_spline is None:
            self._host_spline = NaturalCubicSpline(self._r64.to(self.r.dtype), self._N64.to(self.r.dtype))
        rr = r.to(self.r.dtype)
        value = self._host_spline(rr)
        value = torch.where(rr < self._host_spline.x[0], torch.zeros_like(value), value)
        return torch.where(rr > self._host_spline.x[-1], torch.ones_like(value), value)


__all__ = ["ICDataFile", "MV"]
