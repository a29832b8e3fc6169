"""Batched BK evolution of many parameter sets (one multi-set launch per kernel and stage) and
the request loop: every result equals the same computation run alone."""

from __future__ import annotations

import pytest
import torch

from nlo_bk_optimized_b200.bk.config import IntegrationMethod

pytestmark = pytest.mark.gpu

BK = dict(RPOINTS=63, MINR=1e-6, MAXR=1e2, DE_SOLVER_STEP=0.2, STEPPER="rk4", INTMETHOD_NLO=IntegrationMethod.SOBOL)


def _ics():
    from nlo_bk_optimized_b200 import MV

    return [MV(qs0sqr=0.1), MV(qs0sqr=0.3, gamma=1.2), MV(qs0sqr=0.45, ec=30.0), MV(qs0sqr=0.2, gamma=0.9),
            MV(qs0sqr=0.05, ec=80.0)]


@pytest.mark.parametrize("dtype, rtol", [(torch.float64, 1e-12), (torch.float32, 1e-12)])
def test_batch_equals_individual_solves(dtype, rtol):
    """Five sets with four different budgets (64 r: one CTA group of seven 64-lane slots, two
    of them empty) against solve_bk of each set alone: the same points and the same per-lane
    arithmetic, so the rows agree up to the order of the FP64 sums of the CTA partials
    (1e-12 relative after 3 RK4 steps, in both builds)."""
    from nlo_bk_optimized_b200 import BKConfig, solve_bk
    from nlo_bk_optimized_b200.bk.batch import solve_bk_batch

    ics = _ics()
    budgets = [1 << 10, 1 << 12, 1 << 11, 1 << 12, 1000]
    config = BKConfig(MCINTPOINTS=1 << 10, **BK)
    for waves in (1, 4):
        tables = solve_bk_batch(ics, 0.6, config, samples=budgets, device="cuda", dtype=dtype, waves=waves)
        for ic, budget, table in zip(ics, budgets, tables):
            alone = solve_bk(ic, 0.6, BKConfig(MCINTPOINTS=budget, **BK), device="cuda", dtype=dtype, seed=0)
            assert torch.equal(alone.y, table.y)
            assert alone.N.dtype == table.N.dtype
            torch.testing.assert_close(table.N.double(), alone.N.double(), rtol=rtol, atol=0)
            assert not torch.equal(table.N[-1], table.N[0])


@pytest.mark.parametrize("rpoints, n_sets", [(599, 1), (199, 3), (63, 17)])
def test_batch_layouts(rpoints, n_sets):
    """The CTA layouts of the multi-set launch against solve_bk: 600 r (448-lane slots, one
    set per CTA, two parent tiles per set), 200 r (two 224-lane slots per CTA, the second
    group half empty) and 64 r with 17 sets (three groups of seven slots, four empty)."""
    from nlo_bk_optimized_b200 import MV, BKConfig, solve_bk
    from nlo_bk_optimized_b200.bk.batch import solve_bk_batch

    grid = dict(BK, RPOINTS=rpoints)
    ics = [MV(qs0sqr=0.05 + 0.025 * k) for k in range(n_sets)]
    budgets = [1 << (8 + k % 3) for k in range(n_sets)]
    tables = solve_bk_batch(ics, 0.2, BKConfig(MCINTPOINTS=1 << 9, **grid), samples=budgets, device="cuda",
                            dtype=torch.float64, waves=2)
    for k in sorted({0, n_sets // 2, n_sets - 1}):
        alone = solve_bk(ics[k], 0.2, BKConfig(MCINTPOINTS=budgets[k], **grid), device="cuda", dtype=torch.float64,
                         seed=0)
        torch.testing.assert_close(tables[k].N, alone.N, rtol=1e-12, atol=0)


def test_replayed_set_steps_equal_launched_steps():
    """The multi-set evolution on more than 192 points replays a CUDA graph of one step after
    its first; one-step calls from each previous row give the same rows bit for bit."""
    from nlo_bk_optimized_b200 import BKConfig
    from nlo_bk_optimized_b200.bk.batch import evolve_batch
    from nlo_bk_optimized_b200.bk.evolution import _r_grid

    config = BKConfig(MCINTPOINTS=1 << 10, **dict(BK, RPOINTS=199))
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    N0 = torch.stack([ic.dipole_amplitude(r.cpu()).to(torch.float64) for ic in _ics()]).cuda()
    budgets = [1 << 10, 1 << 12, 1 << 11, 1 << 12, 1000]
    whole = evolve_batch(N0, r, 4, config, budgets, waves=2)
    rows = [N0]
    for _ in range(4):
        rows.append(evolve_batch(rows[-1], r, 1, config, budgets, waves=2)[:, 1])
    assert torch.equal(whole, torch.stack(rows, dim=1))
    assert not torch.equal(whole[:, -1], whole[:, 1])


def test_wave_autotuner_returns_a_choice():
    from nlo_bk_optimized_b200 import MV, BKConfig
    from nlo_bk_optimized_b200.bk.batch import WAVE_CHOICES, tune_waves
    from nlo_bk_optimized_b200.bk.evolution import _r_grid

    config = BKConfig(MCINTPOINTS=1 << 10, **BK)
    r = _r_grid(config, device="cuda", dtype=torch.float64)
    N0 = torch.stack([MV(qs0sqr=q).dipole_amplitude(r.cpu()).to(torch.float64) for q in (0.1, 0.2, 0.3, 0.4)])
    assert tune_waves(N0.cuda(), r, config, [1 << 10] * 4, sample_sets=4) in WAVE_CHOICES


def _requests():
    from nlo_bk_optimized_b200.serving import Request

    return [
        Request(0.2, 1.0, 1.0, ((5.0, 1e-2), (12.0, 3e-2)), 1 << 12, 0),
        Request(0.35, 1.1, 5.0, ((2.0, 5e-2),), 1 << 11, 1),
        Request(0.1, 0.9, 20.0, ((8.0, 2e-2), (3.0, 4e-2), (20.0, 5e-2)), 1 << 12, 2),
        Request(0.2, 1.0, 1.0, ((5.0, 1e-2), (12.0, 3e-2)), 1 << 12, 0),  # same as the first: cached table
    ]


def test_served_results_equal_results_alone():
    """Every served request's table equals its evolution alone to 1e-12 (the evolutions in
    flight advance together through multi-set launches, whose CTA partials add in another
    order), and its structure functions equal the plain single-solve path's to 1e-6: the
    merged DIS launches split the samples of each integral over other CTAs, and the adaptive
    grids carry the FP64 ordering differences (~1e-15) to ~1e-9."""
    from nlo_bk_optimized_b200 import BKConfig
    from nlo_bk_optimized_b200.dis import DISConfig, DISOrder, Quark, QuarkType
    from nlo_bk_optimized_b200.serving import Server, run_alone

    bk = BKConfig(MCINTPOINTS=1 << 10, **BK)
    dis = DISConfig(order=DISOrder.NLO, quarks=(Quark(QuarkType.LIGHT, 0.14),))
    server = Server(bk, dis, slots=8, waves=2)
    requests = _requests()
    futures = [server.submit(req) for req in requests[:3]]
    responses = [f.result(timeout=600) for f in futures]
    responses.append(server.submit(requests[3]).result(timeout=600))  # after the first: its table is resident
    server.close()
    stats = server.stats.summary()
    assert stats["requests"] == 4 and stats["points"] == 8
    assert stats["p50_s"] is not None and stats["p99_s"] >= stats["p50_s"]
    assert responses[3].cached_table
    assert sum(server.batches) == 4
    assert max(server.step_sets) >= 2  # evolutions of different requests advanced in the same launches
    for req, resp in zip(requests, responses):
        alone = run_alone(req, bk, dis)
        torch.testing.assert_close(resp.table.N, alone.table.N, rtol=1e-12, atol=0)
        for key in ("F2", "FL", "FT", "sigma_r"):
            a, b = getattr(alone, key).cpu(), getattr(resp, key).cpu()
            assert torch.allclose(a, b, rtol=1e-6, atol=0), key


def test_merged_dis_batch_over_different_tables_equals_each_alone():
    """structure_functions_many: the points of two tables (each its own seed) in one batch
    equal each table's points run alone."""
    from nlo_bk_optimized_b200 import MV, BKConfig, solve_bk
    from nlo_bk_optimized_b200.dipole import BKDipole
    from nlo_bk_optimized_b200.dis import DISConfig, DISOrder, Quark, QuarkType, structure_functions
    from nlo_bk_optimized_b200.dis import structure_functions_many

    bk = BKConfig(MCINTPOINTS=1 << 10, **BK)
    dis = DISConfig(order=DISOrder.NLO, quarks=(Quark(QuarkType.LIGHT, 0.14),))
    tables = [BKDipole(solve_bk(MV(qs0sqr=q), 8.0, bk, device="cuda", dtype=torch.float64, seed=0))
              for q in (0.15, 0.4)]
    pts = [[(5.0, 1e-2), (12.0, 3e-2)], [(2.0, 5e-2), (8.0, 2e-2), (20.0, 4e-2)]]
    opts = {"vegas_samples": 4096, "vegas_iterations": 4, "vegas_min_iterations": 4}
    Q2 = [q for group in pts for q, _ in group]
    xs = [x for group in pts for _, x in group]
    dipoles = [tables[k] for k, group in enumerate(pts) for _ in group]
    seeds = [7 + k for k, group in enumerate(pts) for _ in group]
    merged = structure_functions_many(Q2, xs, dipoles, dis, sqrt_s=318.0, seeds=seeds, **opts)
    offset = 0
    for k, group in enumerate(pts):
        alone = structure_functions(torch.tensor([q for q, _ in group], dtype=torch.float64),
                                    torch.tensor([x for _, x in group], dtype=torch.float64), tables[k], dis,
                                    sqrt_s=318.0, seed=7 + k, **opts)
        for key in ("F2", "FL", "sigma_r"):
            got = merged[key][offset:offset + len(group)].cpu()
            assert torch.allclose(got, alone[key].cpu(), rtol=1e-6, atol=0), key
        offset += len(group)


def test_admission_never_bypasses_the_memory_check():
    from nlo_bk_optimized_b200 import BKConfig
    from nlo_bk_optimized_b200.dis import DISConfig, DISOrder, Quark, QuarkType
    from nlo_bk_optimized_b200.serving import Server

    total = torch.cuda.get_device_properties(0).total_memory
    bk = BKConfig(MCINTPOINTS=1 << 10, **BK)
    dis = DISConfig(order=DISOrder.NLO, quarks=(Quark(QuarkType.LIGHT, 0.14),))
    server = Server(bk, dis, slots=2, reserve_bytes=total)  # nothing can ever fit
    future = server.submit(_requests()[0])
    with pytest.raises(MemoryError):
        future.result(timeout=60)
    server.close()
