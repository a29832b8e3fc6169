"""BK configuration, initial conditions and the device evolution."""

from nlo_bk_optimized_b200.bk.batch import solve_bk_batch
from nlo_bk_optimized_b200.bk.config import BKConfig, BKOrder, IntegrationMethod
from nlo_bk_optimized_b200.bk.evolution import DNDYResult, bk_steps, compute_dndy, evolve_table, rhs, solve_bk
from nlo_bk_optimized_b200.bk.initial_conditions import MV, ICDataFile
from nlo_bk_optimized_b200.bk.sharded import solve_bk_sharded

__all__ = [
    "BKConfig",
    "BKOrder",
    "DNDYResult",
    "ICDataFile",
    "IntegrationMethod",
    "MV",
    "bk_steps",
    "compute_dndy",
    "evolve_table",
    "rhs",
    "solve_bk",
    "solve_bk_batch",
    "solve_bk_sharded",
]
