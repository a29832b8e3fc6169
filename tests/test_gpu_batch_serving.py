"""Batched BK evolution over CUDA streams and the request loop: every result equals the
same computation run alone."""

from __future__ import annotations

import pytest
import torch

from nlo_bk_optimized_b200.bk.config import IntegrationMethod

pytestmark = pytest.mark.gpu

BK = dict(RPOINTS=63, MINR=1e-6, MAXR=1e2, DE_SOLVER_STEP=0.2, STEPPER="rk4", INTMETHOD_NLO=IntegrationMethod.SOBOL)


def test_batch_equals_individual_solves():
    from nlo_bk_optimized_b200 import MV, BKConfig, solve_bk
    from nlo_bk_optimized_b200.bk.batch import solve_bk_batch

    ics = [MV(qs0sqr=0.1), MV(qs0sqr=0.3, gamma=1.2), MV(qs0sqr=0.45, ec=30.0)]
    budgets = [1 << 10, 1 << 12, 1 << 11]
    config = BKConfig(MCINTPOINTS=1 << 10, **BK)
    tables = solve_bk_batch(ics, 0.6, config, samples=budgets, device="cuda", dtype=torch.float64, streams=3)
    for ic, budget, table in zip(ics, budgets, tables):
        alone = solve_bk(ic, 0.6, BKConfig(MCINTPOINTS=budget, **BK), device="cuda", dtype=torch.float64, seed=0)
        assert torch.equal(alone.y, table.y)
        assert torch.equal(alone.N, table.N)


def test_stream_autotuner_returns_a_choice():
    from nlo_bk_optimized_b200 import MV, BKConfig
    from nlo_bk_optimized_b200.bk.batch import STREAM_CHOICES, tune_streams
    from nlo_bk_optimized_b200.bk.evolution import _r_grid

    config = BKConfig(MCINTPOINTS=1 << 10, **BK)
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    N0 = torch.stack([MV(qs0sqr=q).dipole_amplitude(r.cpu()).to(torch.float64) for q in (0.1, 0.2, 0.3, 0.4)])
    assert tune_streams(N0.cuda(), r, config, [1 << 10] * 4, sample_sets=4) in STREAM_CHOICES


def _requests():
    from nlo_bk_optimized_b200.serving import Request

    return [
        Request(0.2, 1.0, 1.0, ((5.0, 1e-2), (12.0, 3e-2)), 1 << 12, 0),
        Request(0.35, 1.1, 5.0, ((2.0, 5e-2),), 1 << 11, 1),
        Request(0.1, 0.9, 20.0, ((8.0, 2e-2), (3.0, 4e-2), (20.0, 5e-2)), 1 << 12, 2),
        Request(0.2, 1.0, 1.0, ((5.0, 1e-2), (12.0, 3e-2)), 1 << 12, 0),  # same as the first: cached table
    ]


def test_served_results_equal_results_alone():
    from nlo_bk_optimized_b200 import BKConfig
    from nlo_bk_optimized_b200.dis import DISConfig, DISOrder, Quark, QuarkType
    from nlo_bk_optimized_b200.serving import Server, run_alone

    bk = BKConfig(MCINTPOINTS=1 << 10, **BK)
    dis = DISConfig(order=DISOrder.NLO, quarks=(Quark(QuarkType.LIGHT, 0.14),))
    server = Server(bk, dis, slots=3)
    futures = [server.submit(req) for req in _requests()]
    responses = [f.result(timeout=600) for f in futures]
    server.close()
    stats = server.stats.summary()
    assert stats["requests"] == 4 and stats["points"] == 8
    assert stats["p50_s"] is not None and stats["p99_s"] >= stats["p50_s"]
    assert any(r.cached_table for r in responses[1:])
    for req, resp in zip(_requests()[:2], responses[:2]):
        alone = run_alone(req, bk, dis)
        assert torch.equal(alone.table.N, resp.table.N)
        for key in ("F2", "FL", "FT", "sigma_r"):
            a, b = getattr(alone, key).cpu(), getattr(resp, key).cpu()
            assert torch.allclose(a, b, rtol=1e-12, atol=0)
