"""Loaders for the committed golden fixtures (tests/golden/*.npz)."""

from __future__ import annotations

from functools import lru_cache
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


@lru_cache(maxsize=None)
def bk_reference() -> dict[str, np.ndarray]:
    with np.load(GOLDEN / "bk_reference.npz") as data:
        return {key: data[key] for key in data.files}


@lru_cache(maxsize=None)
def bk_table_mc50w() -> dict[str, np.ndarray]:
    with np.load(GOLDEN / "bk_table_mc50w.npz") as data:
        return {key: data[key] for key in data.files}


@lru_cache(maxsize=None)
def bk_variants() -> dict[str, np.ndarray]:
    with np.load(GOLDEN / "bk_variants.npz") as data:
        return {key: data[key] for key in data.files}


def variant_config(name: str):
    """The package's BKConfig for a variant of bk_variants.npz (grid of make_golden.variants)."""
    import ast

    from nlo_bk_optimized_b200.bk import config as bkc

    data = bk_variants()
    names = [str(n) for n in data["names"]]
    kc_names = [str(n) for n in data["kc_names"]]
    if name in names:
        overrides = ast.literal_eval(str(data["overrides"][names.index(name)]))
    else:
        overrides = ast.literal_eval(str(data["kc_overrides"][kc_names.index(name)]))
    kwargs = {}
    for field, value in overrides.items():
        if isinstance(value, str):
            for enum in (bkc.BKOrder, bkc.RunningCouplingLO, bkc.RunningCouplingNLO, bkc.ResummationCoupling):
                if value in enum.__members__:
                    value = enum[value]
                    break
        kwargs[field] = value
    kwargs.setdefault("INTMETHOD_NLO", bkc.IntegrationMethod.SOBOL)  # the oracle's fixed Sobol points
    kwargs.setdefault("STEPPER", "rk4")
    return bkc.BKConfig(RPOINTS=99, MINR=1e-6, MAXR=1e2, **kwargs)


@lru_cache(maxsize=None)
def bk_ic() -> dict[str, np.ndarray]:
    with np.load(GOLDEN / "bk_ic.npz") as data:
        return {key: data[key] for key in data.files}


def synthetic_ic() -> tuple[np.ndarray, np.ndarray]:
    """A 30,000-row tabulated initial condition on the grid of the reference's shipped
    xb_001.dat (log-uniform from 1e-7 to 500): N = 1 - exp(-(r^2 Qs^2)^1.1/4 log(1/(r
    Lambda) + e)) with Qs^2 = 0.104.  bk_ic.npz holds the SHA-256 of its bytes."""
    i = np.arange(30000, dtype=np.float64)
    r = 1e-7 * np.exp(i * (np.log(500.0 / 1e-7) / 29999.0))
    exponent = (r * r * 0.104) ** 1.1 / 4 * np.log(1 / (r * 0.241) + np.e)
    N = -np.expm1(-exponent)
    return r, N


def write_synthetic_ic(path) -> None:
    r, N = synthetic_ic()
    np.savetxt(path, np.stack((r, N), axis=1), fmt="%.17e")
