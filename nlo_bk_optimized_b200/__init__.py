"""B200-native NLO BK evolution with the public entry points of the reference
``nlo_torch`` package (HaowuDuan/nlo_bk_optimized, torch_nlo_clean/src/nlo_torch/__init__.py).

The compute path is libnlo_b200.so (sm_100a CUDA kernels behind a C ABI,
include/nlo_b200.h); this package is the host-side mirror of the reference API.
"""

from nlo_bk_optimized_b200.bk import (
    MV,
    BKConfig,
    BKOrder,
    ICDataFile,
    IntegrationMethod,
    bk_steps,
    compute_dndy,
    evolve_table,
    solve_bk,
    solve_bk_batch,
    solve_bk_sharded,
)
from nlo_bk_optimized_b200.dipole import DipoleTable, load_bk_table, save_bk_table

__all__ = [
    "BKConfig",
    "BKOrder",
    "DipoleTable",
    "ICDataFile",
    "IntegrationMethod",
    "MV",
    "bk_steps",
    "compute_dndy",
    "evolve_table",
    "load_bk_table",
    "save_bk_table",
    "solve_bk",
    "solve_bk_batch",
    "solve_bk_sharded",
]
