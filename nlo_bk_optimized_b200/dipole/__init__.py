"""Dipole amplitudes, tables and the legacy BK text format."""

from nlo_bk_optimized_b200.dipole.amplitude import GBW, AmplitudeInterpolation, BKDipole
from nlo_bk_optimized_b200.dipole.table import DipoleTable, load_bk_table, save_bk_table

__all__ = ["AmplitudeInterpolation", "BKDipole", "DipoleTable", "GBW", "load_bk_table", "save_bk_table"]
