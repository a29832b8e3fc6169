"""BK evolution sharded over the GPUs of one node (one process per GPU).

Rank k of W computes its share of the right-hand side (``nlo_bk_rhs_shard``): K1 of the
parents i with i % W == k (interleaving balances the saturated, inactive parents), and
K2+Kf of every active parent over the k-th W-th of the Sobol indices, divided by the total
sample count.  The ranks sum their rows with one all-reduce of R doubles per stage (3.2 KB
at R = 400, over NCCL), which gives every rank the whole derivative: K1 exactly, K2+Kf up
to the order of the FP64 sums.  Splitting K2+Kf by sample range rather than by parent
keeps every lane of its kernel busy on every rank, and each rank stages only its own
share of the (parent-independent) sample records.  Every rank then forms the stage with
``nlo_bk_stage`` and refits the full spline itself, so the ranks carry identical rows.  The
stage sequence is that of ``nlo_bk_evolve`` (Euler, Kutta RK3 of bk/evolution.py:190-236,
classical RK4).

``shard_steps`` is the device-independent driver: it takes the rank's partial
right-hand side, the all-reduce and the stage combination as functions, which lets the
multi-rank logic run in CPU processes over gloo as well.
"""

from __future__ import annotations

import ctypes
from collections.abc import Callable

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.bk.config import BKConfig, require_fixed_step
from nlo_bk_optimized_b200.dipole.table import DipoleTable

Rhs = Callable[[torch.Tensor], torch.Tensor]
AllReduce = Callable[[torch.Tensor], None]
Stage = Callable[[torch.Tensor, list, list, bool], torch.Tensor]


def shard_steps(N0: torch.Tensor, steps: int, step: float, stepper: str, rhs: Rhs, all_reduce: AllReduce,
                stage: Stage, clamp: bool) -> list[torch.Tensor]:
    """Rows N(Y_0 .. Y_steps) of a stepper whose every derivative is the all-reduced sum of
    the ranks' partial right-hand sides."""

    def f(state: torch.Tensor) -> torch.Tensor:
        k = rhs(state)
        all_reduce(k)
        return k

    rows = [N0]
    N = N0
    h = step
    for _ in range(steps):
        if stepper == "euler":
            k1 = f(N)
            N = stage(N, [k1], [h], clamp)
        elif stepper == "rk3":
            k1 = f(N)
            k2 = f(stage(N, [k1], [0.5 * h], False))
            k3 = f(stage(N, [k1, k2], [-h, 2.0 * h], False))
            N = stage(N, [k1, k2, k3], [h / 6.0, 4.0 * h / 6.0, h / 6.0], clamp)
        elif stepper == "rk4":
            k1 = f(N)
            k2 = f(stage(N, [k1], [0.5 * h], False))
            k3 = f(stage(N, [k2], [0.5 * h], False))
            k4 = f(stage(N, [k3], [h], False))
            N = stage(N, [k1, k2, k3, k4], [h / 6.0, 2.0 * h / 6.0, 2.0 * h / 6.0, h / 6.0], clamp)
        else:
            raise ValueError(f"unknown stepper {stepper}")
        rows.append(N)
    return rows


class ShardedRhs:
    """A rank's share of the right-hand side (``nlo_bk_rhs_shard``, or with Vegas options
    ``nlo_bk_rhs_vegas``) and the stage combination (``nlo_bk_stage``) on its device, as the
    functions ``shard_steps`` takes.  A Vegas integral needs all of one parent's samples for
    its grid, so with Vegas the rank takes K1 and K2+Kf of its own parents (i % W == k) and
    keeps their grids from stage to stage."""

    def __init__(self, params, r: torch.Tensor, dirs, samples: int, box, rank: int, world: int,
                 workspace: torch.Tensor, status: torch.Tensor, stream, vegas=None) -> None:
        self.lib = _native.load()
        self.params, self.r, self.dirs, self.samples, self.box = params, r, dirs, int(samples), box
        self.rank, self.world = rank, world
        self.workspace, self.status = workspace, status
        self.stream = stream if isinstance(stream, int) or stream is None else stream.cuda_stream
        self.vegas = vegas
        if vegas is not None:
            from nlo_bk_optimized_b200.bk.evolution import vegas_state

            self.grids = vegas_state(r.device, r.numel())

    def rhs(self, N: torch.Tensor) -> torch.Tensor:
        out = torch.empty_like(N)
        if self.vegas is not None:
            _native.check(self.lib.nlo_bk_rhs_vegas(self.params, self.r.data_ptr(), self.r.numel(), None,
                                                    N.data_ptr(), 1, self.rank, self.world, self.vegas, self.dirs,
                                                    self.box, self.grids.data_ptr(), out.data_ptr(), None, None,
                                                    self.workspace.data_ptr(), self.workspace.numel(), self.stream))
            return out
        _native.check(self.lib.nlo_bk_rhs_shard(self.params, self.r.data_ptr(), N.data_ptr(), self.r.numel(),
                                                self.rank, self.world, self.dirs, self.samples, self.box,
                                                out.data_ptr(), self.workspace.data_ptr(), self.workspace.numel(),
                                                self.stream))
        return out

    def stage(self, N: torch.Tensor, ks: list, coefs: list, clamp: bool) -> torch.Tensor:
        out = torch.empty_like(N)
        kp = (ctypes.c_void_p * len(ks))(*[k.data_ptr() for k in ks])
        cf = (ctypes.c_double * len(coefs))(*coefs)
        # like nlo_bk_evolve, only the completed step is clamped and checked
        _native.check(self.lib.nlo_bk_stage(N.data_ptr(), kp, cf, len(ks), self.r.numel(), int(clamp),
                                            out.data_ptr(), self.status.data_ptr() if clamp else None, self.stream))
        return out


def solve_bk_sharded(initial_condition, maxy: float, config: BKConfig = BKConfig(), *,
                     device: torch.device | str | None = None, dtype: torch.dtype = torch.float32, seed: int = 0,
                     group: "torch.distributed.ProcessGroup | None" = None) -> DipoleTable:
    """``solve_bk`` across the ranks of ``group`` (torch.distributed, NCCL for CUDA)."""
    import torch.distributed as dist

    from nlo_bk_optimized_b200.bk.evolution import (
        _r_grid,
        _steps_to,
        initial_row,
        nlo_box,
        params_of,
        precision_of,
        vegas_evolution_setup,
        workspace,
    )

    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if device.type != "cuda":
        raise ValueError("the sharded evolution runs on CUDA devices only")
    params = params_of(config, precision_of(config, dtype))
    r_host = _r_grid(config, device="cpu", dtype=torch.float64)
    N0 = initial_row(initial_condition, r_host, device).contiguous()
    r = r_host.to(device)
    points = r.numel()
    lower, width = nlo_box(float(r_host[0]), float(r_host[-1]))
    box = _native.box(lower, width)
    vegas, dirs_all = vegas_evolution_setup(config, seed)
    ws = workspace(device, points, vegas)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    stream = _native.stream_handle(device)
    ys = _steps_to(0.0, maxy, config.DE_SOLVER_STEP)
    steps = len(ys)
    clamp = bool(config.FORCE_POSITIVE_N)

    if config.KINEMATICAL_CONSTRAINT:
        raise ValueError("the sharded evolution has no kinematical constraint (it reads no amplitude history)")
    require_fixed_step(config, "the sharded evolution")
    sharded = ShardedRhs(params, r, dirs_all if vegas is not None else dirs_all[0], int(config.MCINTPOINTS), box,
                         rank, world, ws, status, stream, vegas=vegas)

    def all_reduce(k: torch.Tensor) -> None:
        if world > 1:
            dist.all_reduce(k, op=dist.ReduceOp.SUM, group=group)

    with torch.cuda.device(device):
        rows = shard_steps(N0, steps, config.DE_SOLVER_STEP, config.stepper, sharded.rhs, all_reduce,
                           sharded.stage, clamp)
        if int(status.item()) != 0:
            raise FloatingPointError("non-finite BK amplitude during the rapidity evolution")
    y = torch.tensor([0.0, *ys], dtype=dtype, device=device)
    N = torch.stack(rows)
    return DipoleTable(r=r.to(dtype), y=y, N=N.to(dtype), x0=initial_condition.x0)


__all__ = ["ShardedRhs", "shard_steps", "solve_bk_sharded"]
