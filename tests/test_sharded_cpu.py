"""The multi-rank BK evolution driver (nlo_bk_optimized_b200/bk/sharded.py) over gloo on
CPU, world size 2: each rank supplies the oracle's shard right-hand side (K1 of its own
parents i % 2 == rank, K2+Kf of every active parent over its half of the Sobol points),
and the driver's all-reduce and stage sequence must reproduce the single-process oracle
evolution."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from nlo_bk_optimized_b200.bk.config import BKConfig
from nlo_bk_optimized_b200.bk.sharded import shard_steps

R_POINTS, SAMPLES, STEP, STEPS = 23, 128, 0.2, 2


def problem():
    config = BKConfig(RPOINTS=R_POINTS, MINR=1e-6, MAXR=1e2, MCINTPOINTS=SAMPLES, DE_SOLVER_STEP=STEP)
    r = oracle.r_grid(1e-6, 1e2, R_POINTS)
    N0 = oracle.mv_amplitude(r, 0.2)
    phys = oracle.physics(config)
    state, shift = oracle.sobol_state(4, 0)
    pts = oracle.sobol(state, shift, 0, SAMPLES, as_f32=True)
    return r, N0, phys, pts


def stage_torch(N, ks, coefs, clamp):
    out = N.clone()
    for k, c in zip(ks, coefs):
        out = out + c * k
    return out.clamp(0, 1) if clamp else out


def _worker(rank, world, port, stepper, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, N0, phys, pts = problem()

        def rhs(N):
            return torch.from_numpy(oracle.derivative_shard(N.numpy(), r, phys, pts, True, rank, world))

        rows = shard_steps(torch.from_numpy(N0.copy()), STEPS, STEP, stepper, rhs,
                           lambda k: dist.all_reduce(k, op=dist.ReduceOp.SUM), stage_torch, True)
        results[rank] = torch.stack(rows).numpy()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("stepper", ["rk4", "rk3", "euler"])
def test_two_rank_evolution_matches_single_process(stepper):
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    results = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, 2, port, stepper, results)) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    r, N0, phys, pts = problem()
    ys, ref = oracle.evolve(N0, r, phys, pts, True, STEP, STEP * STEPS, stepper)
    for rank in range(2):
        got = results[rank]
        assert got.shape == ref.shape
        assert np.max(np.abs(got - ref)) < 1e-12
    assert np.array_equal(results[0], results[1])


def test_shard_parts_add_up_to_the_whole_derivative():
    r, N0, phys, pts = problem()
    whole = oracle.derivative(N0, r, phys, pts, True).dNdy
    for shards in (2, 3, 5):
        total = sum(oracle.derivative_shard(N0, r, phys, pts, True, k, shards) for k in range(shards))
        assert np.max(np.abs(total - whole) / np.maximum(np.abs(whole), 1e-300)) < 1e-12
