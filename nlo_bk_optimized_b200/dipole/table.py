"""BK amplitude tables and the legacy text format the C++ solver writes.

``DipoleTable`` keeps the interface of the reference's table type
(torch_nlo_clean/src/nlo_torch/dipole/table.py:12-45): amplitudes ``N[len(y), len(r)]``
on a positive, increasing r grid at increasing rapidities, with the ``x0`` the table
starts from.  ``load_bk_table`` / ``save_bk_table`` read and write the text format of
the C++ ``nlobk`` solver (the shipped ``xb_001_mc50w.dat``; the reference's reader and
writer are dipole/table.py:48-144).

The format, as this module implements it:

* lines are stripped; blank lines and comments (``#`` not followed by ``##``) are ignored;
* a *directive* is a line ``###<number>``;
* the first four directives describe the grid: the smallest r, the ratio of consecutive
  r, the number of r points and x0, so r_i = minr * ratio**i;
* every further directive opens a block at rapidity ``<number>``, followed by exactly one
  amplitude per r point, one per line.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch


def _problems(table: "DipoleTable"):
    """Yield (exception type, message) for the first rule the table breaks; the rules are
    checked in order and the later ones assume the earlier hold."""
    r, y, N = table.r, table.y, table.N
    rules = (
        (lambda: r.ndim == 1 and y.ndim == 1 and N.ndim == 2, ValueError,
         "expected one-dimensional r and y and a two-dimensional N"),
        (lambda: r.numel() >= 2 and y.numel() >= 1, ValueError, "a table needs at least 2 r points and 1 rapidity"),
        (lambda: tuple(N.shape) == (y.numel(), r.numel()), ValueError,
         f"N has shape {tuple(N.shape)}; expected (len(y), len(r)) = ({y.numel()}, {r.numel()})"),
        (lambda: r.device == y.device == N.device, ValueError, "r, y and N live on different devices"),
        (lambda: r.dtype == y.dtype == N.dtype, ValueError, "r, y and N have different dtypes"),
        (lambda: r.is_floating_point(), TypeError, "r, y and N must be floating point"),
        (lambda: bool(torch.isfinite(r).all()), ValueError, "r has a non-finite value"),
        (lambda: bool(torch.isfinite(y).all()), ValueError, "y has a non-finite value"),
        (lambda: bool(torch.isfinite(N).all()), ValueError, "N has a non-finite value"),
        (lambda: bool((r > 0).all()) and bool((r.diff() > 0).all()), ValueError,
         "r must be positive and strictly increasing"),
        (lambda: y.numel() == 1 or bool((y.diff() > 0).all()), ValueError, "y must be strictly increasing"),
        (lambda: math.isfinite(table.x0) and table.x0 > 0, ValueError, "x0 must be a positive finite number"),
    )
    for holds, kind, message in rules:
        if not holds():
            yield kind, message
            return


@dataclass(frozen=True, slots=True)
class DipoleTable:
    """BK amplitudes ``N(y, r)`` stored at evolution rapidities ``y``."""

    r: torch.Tensor
    y: torch.Tensor
    N: torch.Tensor
    x0: float

    def __post_init__(self) -> None:
        for kind, message in _problems(self):
            raise kind(f"invalid dipole table: {message}")


def _directive(line: str) -> str | None:
    return line[3:].strip() if line.startswith("###") else None


def _number(text: str, what: str, source: Path) -> float:
    try:
        return float(text)
    except ValueError:
        raise ValueError(f"{source}: {what} {text!r} is not a number") from None


def load_bk_table(
    path: str | Path,
    *,
    dtype: torch.dtype = torch.float64,
    device: torch.device | str | None = None,
) -> DipoleTable:
    """Read a table in the C++ solver's text format (see the module docstring)."""

    source = Path(path)
    directives: list[tuple[int, str]] = []  # (position in `values`, text)
    values: list[str] = []
    for raw in source.read_text(encoding="utf-8").splitlines():
        line = raw.strip()
        if not line:
            continue
        text = _directive(line)
        if text is not None:
            directives.append((len(values), text))
        elif not line.startswith("#"):
            values.append(line)
    if len(directives) < 4:
        raise ValueError(f"{source}: expected four grid directives (minr, ratio, points, x0)")
    grid, blocks = directives[:4], directives[4:]
    if grid[-1][0] != 0 or (blocks and blocks[0][0] != 0) or (not blocks and values):
        raise ValueError(f"{source}: amplitude values before the first rapidity directive")
    minr = _number(grid[0][1], "minr", source)
    ratio = _number(grid[1][1], "r ratio", source)
    count = _number(grid[2][1], "number of r points", source)
    x0 = _number(grid[3][1], "x0", source)
    if not (minr > 0 and ratio > 1 and count >= 2 and count == int(count) and x0 > 0):
        raise ValueError(f"{source}: grid directives out of range (minr {minr}, ratio {ratio}, points {count}, "
                         f"x0 {x0})")
    points = int(count)
    if not blocks:
        raise ValueError(f"{source}: no rapidity blocks")
    # each block's values run from its directive to the next one
    bounds = [start for start, _ in blocks] + [len(values)]
    for k, (start, stop) in enumerate(zip(bounds[:-1], bounds[1:])):
        if stop - start != points:
            raise ValueError(f"{source}: rapidity block {k} holds {stop - start} amplitudes, expected {points}")
    ys = [_number(text, "rapidity", source) for _, text in blocks]
    try:
        amplitudes = np.asarray(values, dtype=np.float64).reshape(len(blocks), points)
    except ValueError:
        bad = next(v for v in values if not _is_float(v))
        raise ValueError(f"{source}: amplitude {bad!r} is not a number") from None
    exponent = torch.arange(points, dtype=dtype, device=device)
    r = minr * torch.pow(torch.tensor(ratio, dtype=dtype, device=device), exponent)
    return DipoleTable(
        r=r,
        y=torch.tensor(ys, dtype=dtype, device=device),
        N=torch.as_tensor(amplitudes, device=device).to(dtype),
        x0=x0,
    )


def _is_float(text: str) -> bool:
    try:
        float(text)
        return True
    except ValueError:
        return False


def save_bk_table(path: str | Path, table: DipoleTable) -> None:
    """Write ``table`` in the C++ solver's text format, 15-digit mantissas.

    The format stores the grid as (minr, ratio), so the grid must be logarithmically
    uniform.  A float64 grid is written with ratio r[1]/r[0] and checked to 2e-12.  A
    float32 grid is the float64 grid rounded once (solve_bk forms it in float64): its
    r[1]/r[0] is off by about 1e-7, which the 100th power turns into 1e-5, so its ratio is
    taken from the end points in float64 instead and checked to 5e-6; the header then
    reproduces the grid to float32 rounding."""

    r = table.r.detach().to("cpu", torch.float64)
    if table.r.dtype == torch.float32:
        ratio = float((r[-1] / r[0]) ** (1.0 / (r.numel() - 1)))
        tolerance = 5e-6
    else:
        ratio = float(r[1] / r[0])
        tolerance = 2e-12
    rebuilt = float(r[0]) * ratio ** np.arange(r.numel(), dtype=np.float64)
    if not np.allclose(r.numpy(), rebuilt, rtol=tolerance, atol=0.0):
        raise ValueError("the legacy BK format stores (minr, ratio): the r grid must be logarithmically uniform")
    y = table.y.detach().to("cpu", torch.float64).numpy()
    N = table.N.detach().to("cpu", torch.float64).numpy()
    header = ["# nlo_bk_optimized_b200 BK dipole table",
              *(f"###{v:.15e}" for v in (float(r[0]), ratio)), f"###{r.numel()}", f"###{table.x0:.15e}"]
    body = []
    for rapidity, row in zip(y, N):
        body.append(f"###{rapidity:.15e}")
        body.extend(f"{v:.15e}" for v in row)
    Path(path).write_text("\n".join(header + body) + "\n", encoding="utf-8")


__all__ = ["DipoleTable", "load_bk_table", "save_bk_table"]
