"""Direct access to the individual device operators of libnlo_b200.so.

These wrap one C-ABI entry point each (include/nlo_b200.h) on torch-allocated
device buffers and the current CUDA stream; the parity tests call them to
compare each stage with the oracle on identical inputs.
"""

from __future__ import annotations

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.bk.config import BKConfig
from nlo_bk_optimized_b200.bk.evolution import nlo_box, params_of, precision_of


def sobol_draw(dims: int, seed: int, n: int, *, offset: int = 0, dtype: torch.dtype = torch.float32,
               device: torch.device | str = "cuda") -> torch.Tensor:
    """Points offset..offset+n-1 of SobolEngine(dims, scramble=True, seed) drawn on the device."""

    device = torch.device(device)
    out = torch.empty((n, dims), dtype=dtype, device=device)
    precision = _native.PRECISION_FP64 if dtype == torch.float64 else _native.PRECISION_MIXED
    lib = _native.load()
    with torch.cuda.device(device):
        _native.check(lib.nlo_sobol_draw(_native.sobol_dirs(dims, seed), offset, n, precision,
                                         out.data_ptr(), _native.stream_handle(device)))
    return out


def splines(r: torch.Tensor, N: torch.Tensor, *, force_positive: bool = True) -> dict[str, torch.Tensor]:
    """log N and log S natural-spline coefficients (float64) of one amplitude row."""

    _native.require_cuda(r, "r")
    r64 = r.to(torch.float64).contiguous()
    N64 = N.to(device=r.device, dtype=torch.float64).contiguous()
    n = r64.numel()
    lib = _native.load()
    out = torch.empty(int(lib.nlo_bk_spline_doubles(n)), dtype=torch.float64, device=r.device)
    with torch.cuda.device(r.device):
        _native.check(lib.nlo_bk_splines(r64.data_ptr(), N64.data_ptr(), n, int(force_positive), out.data_ptr(),
                                         _native.stream_handle(r.device)))
    coef = out[n:n + 8 * (n - 1)].view(2, n - 1, 4)
    return {"x": out[:n], "n": coef[0], "s": coef[1], "raw": out}


def active(N: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    _native.require_cuda(N, "N")
    N64 = N.to(torch.float64).contiguous()
    n = N64.numel()
    idx = torch.empty(n, dtype=torch.int32, device=N.device)
    count = torch.empty(1, dtype=torch.int32, device=N.device)
    lib = _native.load()
    with torch.cuda.device(N.device):
        _native.check(lib.nlo_bk_active(N64.data_ptr(), n, idx.data_ptr(), count.data_ptr(),
                                        _native.stream_handle(N.device)))
    return idx, count


def k1(r: torch.Tensor, N: torch.Tensor, config: BKConfig = BKConfig(), *, precision: int | None = None) -> torch.Tensor:
    """K1 of every active parent by the fixed rule (float64 [R], zeros elsewhere)."""

    sp = splines(r, N, force_positive=config.FORCE_POSITIVE_N)
    idx, count = active(N)
    prec = precision if precision is not None else precision_of(config, r.dtype)
    out = torch.empty(r.numel(), dtype=torch.float64, device=r.device)
    lib = _native.load()
    r64 = r.to(torch.float64).contiguous()
    with torch.cuda.device(r.device):
        _native.check(lib.nlo_bk_k1(params_of(config, prec), r64.data_ptr(), r64.numel(), sp["raw"].data_ptr(),
                                    idx.data_ptr(), count.data_ptr(), out.data_ptr(), _native.stream_handle(r.device)))
    return out


def k2kf(r: torch.Tensor, N: torch.Tensor, config: BKConfig = BKConfig(), *, samples: int | None = None,
         offset: int = 0, seed: int = 0, precision: int | None = None) -> torch.Tensor:
    """Per-parent [sum w K2, sum w Kf, sum w^2 (K2+Kf)^2] over Sobol points offset.. (float64 [R, 3])."""

    sp = splines(r, N, force_positive=config.FORCE_POSITIVE_N)
    idx, count = active(N)
    prec = precision if precision is not None else precision_of(config, r.dtype)
    r64 = r.to(torch.float64).contiguous()
    n = r64.numel()
    out = torch.empty((n, 3), dtype=torch.float64, device=r.device)
    lib = _native.load()
    ws = torch.empty(int(lib.nlo_bk_k2kf_workspace_bytes(n)), dtype=torch.uint8, device=r.device)
    lower, width = nlo_box(float(r64[0]), float(r64[-1]))
    with torch.cuda.device(r.device):
        _native.check(lib.nlo_bk_k2kf(params_of(config, prec), r64.data_ptr(), n, sp["raw"].data_ptr(),
                                      idx.data_ptr(), count.data_ptr(), _native.sobol_dirs(4, seed), offset,
                                      int(config.MCINTPOINTS if samples is None else samples),
                                      _native.box(lower, width), out.data_ptr(), ws.data_ptr(), ws.numel(),
                                      _native.stream_handle(r.device)))
    return out


__all__ = ["active", "k1", "k2kf", "sobol_draw", "splines"]
