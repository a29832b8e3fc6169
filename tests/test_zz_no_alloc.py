"""The allocation-free K2+Kf entry point (nlo_bk_k2kf_static).

Some callers cannot let this library allocate device memory -- e.g. a plugin in a
framework that owns the GPU's memory pool, or a serving loop that must not pay
cudaMalloc's latency and implicit synchronisation per request.  For them
nlo_bk_k2kf_static keeps its scratch in a fixed device array instead of a
caller workspace.  This test calls it through the C ABI twice in a row (the
second call reuses the array with the first call's contents) and checks both
results against nlo_bk_k2kf with a workspace, within the FP64 summation-order
tolerance (the two use different CTA counts, so the partial sums are added in a
different order).  It lives in its own file so that pytest collects it last.
"""

from __future__ import annotations

import ctypes

import pytest
import torch

from nlo_bk_optimized_b200 import MV, BKConfig, _native, kernels
from nlo_bk_optimized_b200.bk.evolution import _r_grid, nlo_box, params_of

pytestmark = pytest.mark.gpu


def _inputs(rpoints: int):
    config = BKConfig(RPOINTS=rpoints, MINR=1e-7, MAXR=1e2)
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    N = MV(qs0sqr=0.4).dipole_amplitude(r)
    sp = kernels.splines(r, N)
    idx, count = kernels.active(N)
    lower, width = nlo_box(float(r[0]), float(r[-1]))
    return config, r, sp["raw"], idx, count, _native.box(lower, width)


@pytest.mark.parametrize("precision", [_native.PRECISION_MIXED, _native.PRECISION_FP64])
def test_static_entry_point_matches_workspace_entry_point(precision):
    lib = _native.load()
    config, r, spline, idx, count, box = _inputs(399)
    n = r.numel()
    params = params_of(config, precision)
    dirs = _native.sobol_dirs(4, 0)
    samples = 1 << 14
    stream = torch.cuda.current_stream().cuda_stream

    reference = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    ws = torch.empty(int(lib.nlo_bk_k2kf_workspace_bytes(n)), dtype=torch.uint8, device="cuda")
    assert lib.nlo_bk_k2kf(params, r.data_ptr(), n, spline.data_ptr(), idx.data_ptr(), count.data_ptr(), dirs, 0,
                           samples, box, reference.data_ptr(), ws.data_ptr(), ws.numel(), stream) == 0

    outs = [torch.full((n, 3), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    # The first call on a device makes the driver load the code module that holds the fixed
    # array (it stays resident until exit); measure free memory after that warm-up call.
    warm = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    assert lib.nlo_bk_k2kf_static(params, r.data_ptr(), n, spline.data_ptr(), idx.data_ptr(), count.data_ptr(),
                                  dirs, 0, samples, box, warm.data_ptr(), ctypes.c_void_p(stream)) == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]  # driver-level free bytes, not the caching allocator's
    for out in outs:
        code = lib.nlo_bk_k2kf_static(params, r.data_ptr(), n, spline.data_ptr(), idx.data_ptr(), count.data_ptr(),
                                      dirs, 0, samples, box, out.data_ptr(), ctypes.c_void_p(stream))
        assert code == 0, lib.nlo_last_error().decode()
        torch.cuda.synchronize()
    # the property the entry point exists for: nothing was allocated on the device
    assert torch.cuda.mem_get_info()[0] == free_before
    for out in outs:
        torch.testing.assert_close(out, reference, rtol=1e-12, atol=0.0)


def test_static_entry_point_rejects_grids_beyond_its_limit():
    lib = _native.load()
    config, r, spline, idx, count, box = _inputs(599)  # 600 points > 512
    out = torch.empty((r.numel(), 3), dtype=torch.float64, device="cuda")
    code = lib.nlo_bk_k2kf_static(params_of(config, _native.PRECISION_MIXED), r.data_ptr(), r.numel(),
                                  spline.data_ptr(), idx.data_ptr(), count.data_ptr(), _native.sobol_dirs(4, 0), 0,
                                  1024, box, out.data_ptr(), None)
    assert code == 1
    assert b"512" in lib.nlo_last_error()


def test_static_entry_point_rejects_what_the_workspace_entry_point_rejects():
    lib = _native.load()
    config, r, spline, idx, count, box = _inputs(99)
    out = torch.empty((r.numel(), 3), dtype=torch.float64, device="cuda")
    for field, value in (("order", 9), ("rc_lo", -1), ("resum_rc", 7)):
        params = params_of(config, _native.PRECISION_MIXED)
        setattr(params, field, value)
        code = lib.nlo_bk_k2kf_static(params, r.data_ptr(), r.numel(), spline.data_ptr(), idx.data_ptr(),
                                      count.data_ptr(), _native.sobol_dirs(4, 0), 0, 1024, box, out.data_ptr(), None)
        assert code == 1, field
