"""Device pieces of the sharded BK evolution on one GPU: the shard right-hand sides sum
to the full right-hand side, and the single-rank sharded driver reproduces solve_bk."""

from __future__ import annotations

import ctypes

import pytest
import torch

from nlo_bk_optimized_b200.bk.config import IntegrationMethod

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_shard_rhs_sum_to_full_rhs(precision):
    from nlo_bk_optimized_b200 import MV, BKConfig, _native
    from nlo_bk_optimized_b200.bk.evolution import _r_grid, nlo_box, params_of, rhs, workspace

    config = BKConfig(RPOINTS=99, MINR=1e-6, MAXR=1e2, MCINTPOINTS=1 << 12, PRECISION=precision,
                      INTMETHOD_NLO=IntegrationMethod.SOBOL)
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    N = MV(qs0sqr=0.2).dipole_amplitude(r.cpu()).to("cuda", torch.float64)
    full, _, _ = rhs(N, r, config, seed=0)
    lib = _native.load()
    code = _native.PRECISION_FP64 if precision == "fp64" else _native.PRECISION_MIXED
    params = params_of(config, code)
    lower, width = nlo_box(float(r[0]), float(r[-1]))
    ws = workspace(r.device, r.numel())
    for shards in (2, 3):
        total = torch.zeros_like(N)
        for shard in range(shards):
            out = torch.empty_like(N)
            _native.check(lib.nlo_bk_rhs_shard(params, r.data_ptr(), N.data_ptr(), r.numel(), shard, shards,
                                               _native.sobol_dirs(4, 0), config.MCINTPOINTS,
                                               _native.box(lower, width), out.data_ptr(), ws.data_ptr(), ws.numel(),
                                               _native.stream_handle(r.device)))
            total += out
        # K1 is split exactly; K2+Kf's sums over the shards' point ranges are added in another
        # order (the mixed build's FP32 partial sums also group the samples differently)
        scale = full.abs() + 1e-9 * full.abs().max()
        rel = ((total - full).abs() / scale).max()
        assert float(rel) < (1e-12 if precision == "fp64" else 1e-6)


@pytest.mark.parametrize("method", ["SOBOL", "VEGAS"])
def test_single_rank_sharded_driver_matches_solve_bk(method):
    from nlo_bk_optimized_b200 import MV, BKConfig, solve_bk
    from nlo_bk_optimized_b200.bk.sharded import solve_bk_sharded

    config = BKConfig(RPOINTS=63, MINR=1e-6, MAXR=1e2, MCINTPOINTS=1 << 11, DE_SOLVER_STEP=0.2, STEPPER="rk4",
                      INTMETHOD_NLO=IntegrationMethod[method],
                      PRECISION="fp64")
    a = solve_bk(MV(qs0sqr=0.2), 0.4, config, device="cuda", dtype=torch.float64, seed=0)
    b = solve_bk_sharded(MV(qs0sqr=0.2), 0.4, config, device="cuda", dtype=torch.float64, seed=0)
    assert torch.equal(a.y, b.y)
    rel = ((a.N - b.N).abs() / a.N.abs().clamp_min(1e-300)).max()
    assert float(rel) < 1e-12


def test_stage_entry_point():
    from nlo_bk_optimized_b200 import _native

    lib = _native.load()
    N = torch.tensor([0.1, 0.5, 0.9], dtype=torch.float64, device="cuda")
    k1 = torch.tensor([1.0, 1.0, 1.0], dtype=torch.float64, device="cuda")
    k2 = torch.tensor([0.0, -2.0, 4.0], dtype=torch.float64, device="cuda")
    out = torch.empty_like(N)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    kp = (ctypes.c_void_p * 2)(k1.data_ptr(), k2.data_ptr())
    cf = (ctypes.c_double * 2)(0.5, 0.25)
    _native.check(lib.nlo_bk_stage(N.data_ptr(), kp, cf, 2, 3, 1, out.data_ptr(), status.data_ptr(),
                                   _native.stream_handle(N.device)))
    assert out.tolist() == [0.6, 0.5, 1.0]
    assert int(status) == 0
