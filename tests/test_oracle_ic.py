"""The tabulated initial condition (ICDataFile, bk/initial_conditions.py:38-91) on a
30,000-row table: the oracle's natural spline and the package's host path reproduce the
reference's coefficients and amplitudes (tests/golden/bk_ic.npz, made by
tests/golden/make_golden.py ic)."""

from __future__ import annotations

import hashlib

import numpy as np
import torch

import oracle
from golden_data import bk_ic, synthetic_ic, write_synthetic_ic
from nlo_bk_optimized_b200.bk.initial_conditions import ICDataFile


def test_synthetic_table_is_the_one_the_fixture_was_made_from():
    r, N = synthetic_ic()
    assert hashlib.sha256(r.tobytes() + N.tobytes()).hexdigest() == str(bk_ic()["ic_sha256"])


def test_oracle_spline_coefficients_equal_the_reference():
    g = bk_ic()
    r, N = synthetic_ic()
    a, b, c, d = oracle.natural_spline(r, N)
    idx = g["ic_coef_index"]
    # the same FP64 operations in the same order: equal to the bit
    for name, mine in (("a", a), ("b", b), ("c", c), ("d", d)):
        np.testing.assert_array_equal(mine[idx], g[f"ic_{name}"], err_msg=name)


def test_host_path_reads_the_file_and_matches_the_reference(tmp_path):
    g = bk_ic()
    path = tmp_path / "ic.dat"
    write_synthetic_ic(path)
    ic = ICDataFile(path, x0=0.01)
    assert ic.r.numel() == 30000 and ic.min_r == 1e-7
    got = ic.dipole_amplitude(torch.tensor(g["ic_points"])).numpy()
    np.testing.assert_array_equal(got, g["ic_N"])
