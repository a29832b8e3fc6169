"""The tabulated initial condition on the device (nlo_ic_spline / nlo_ic_evaluate): the
30,000-row natural spline is fitted and evaluated on the GPU with the reference's FP64
operations, so its coefficients and amplitudes equal the reference's to the bit
(tests/golden/bk_ic.npz), and the evolution starts from that row."""

from __future__ import annotations

import time

import numpy as np
import pytest
import torch

from golden_data import bk_ic, synthetic_ic, write_synthetic_ic
from nlo_bk_optimized_b200 import BKConfig, _native, solve_bk
from nlo_bk_optimized_b200.bk.config import IntegrationMethod
from nlo_bk_optimized_b200.bk.evolution import _r_grid, compute_dndy
from nlo_bk_optimized_b200.bk.initial_conditions import ICDataFile

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ic_file(tmp_path_factory):
    path = tmp_path_factory.mktemp("ic") / "ic.dat"
    write_synthetic_ic(path)
    return path


def test_device_spline_coefficients_equal_the_reference(ic_file):
    g = bk_ic()
    ic = ICDataFile(ic_file, x0=0.01)
    spline = ic.device_spline("cuda").cpu().numpy()
    n = 30000
    x, a, b, c, d = (spline[:n], spline[n:2 * n - 1], spline[2 * n - 1:3 * n - 2], spline[3 * n - 2:4 * n - 3],
                     spline[4 * n - 3:])
    np.testing.assert_array_equal(x, synthetic_ic()[0])
    idx = g["ic_coef_index"]
    for name, mine in (("a", a), ("b", b), ("c", c), ("d", d)):
        np.testing.assert_array_equal(mine[idx], g[f"ic_{name}"], err_msg=name)


def test_device_amplitude_equals_the_reference(ic_file):
    g = bk_ic()
    ic = ICDataFile(ic_file, x0=0.01)
    got = ic.device_amplitude(torch.tensor(g["ic_points"], device="cuda")).cpu().numpy()
    np.testing.assert_array_equal(got, g["ic_N"])
    # CUDA tensors in the public call take the device path and keep the IC's dtype
    f32 = ICDataFile(ic_file, x0=0.01, dtype=torch.float32)
    out = f32.dipole_amplitude(torch.tensor(g["ic_points"], device="cuda"))
    assert out.dtype == torch.float32 and out.is_cuda


def test_evolution_starts_from_the_device_row(ic_file):
    g = bk_ic()
    config = BKConfig(RPOINTS=399, MINR=1e-7, MAXR=1e2, MCINTPOINTS=256, DE_SOLVER_STEP=0.1,
                      INTMETHOD_NLO=IntegrationMethod.SOBOL)
    table = solve_bk(ICDataFile(ic_file, x0=0.01), 0.1, config, device="cuda", dtype=torch.float64, seed=0)
    grid = _r_grid(config, device="cpu", dtype=torch.float64).numpy()
    np.testing.assert_array_equal(grid, g["ic_points"][:400])
    np.testing.assert_array_equal(table.N[0].cpu().numpy(), g["ic_N"][:400])
    res = compute_dndy(ICDataFile(ic_file, x0=0.01), config, device="cuda", dtype=torch.float64, seed=0)
    assert res.r.numel() > 100 and bool(torch.isfinite(res.K1).all())


def test_fit_time_of_the_30000_row_table(ic_file):
    """One-thread Thomas sweeps: about a millisecond, once per evolution."""
    lib = _native.load()
    r, N = (torch.tensor(v, device="cuda") for v in synthetic_ic())
    out = torch.empty(int(lib.nlo_ic_spline_doubles(30000)), dtype=torch.float64, device="cuda")
    stream = _native.stream_handle(torch.device("cuda"))
    for _ in range(3):
        _native.check(lib.nlo_ic_spline(r.data_ptr(), N.data_ptr(), 30000, out.data_ptr(), stream))
    torch.cuda.synchronize()
    start = time.perf_counter()
    for _ in range(10):
        _native.check(lib.nlo_ic_spline(r.data_ptr(), N.data_ptr(), 30000, out.data_ptr(), stream))
    torch.cuda.synchronize()
    per_fit = (time.perf_counter() - start) / 10
    print(f"nlo_ic_spline, 30000 rows: {per_fit * 1e3:.3f} ms")
    assert per_fit < 0.05
