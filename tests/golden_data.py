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
