"""A request loop for BK tables and DIS structure functions with continuous batching.

A request is one initial-condition parameter set, a list of (Q^2, x_Bj) points and a
Monte Carlo budget.  The server keeps evolved N(Y, r) tables resident on the device in an
LRU cache keyed by the parameter set and budget, admits queued requests whenever a slot
is free and the device has the memory the request needs, and runs every admitted request
on its own CUDA stream, so the kernels of requests that arrived at different times
overlap on the GPU: a request that arrives while others are running starts at once
instead of waiting for the batch.  Each request's work -- ``nlo_bk_evolve`` for its table
(unless cached), then ``structure_functions`` for its points -- is the same computation
as when it runs alone, so its results do not depend on what else is in flight.

Latency is measured per request from ``submit`` to completion; ``stats`` reports
p50/p99 and the point throughput.
"""

from __future__ import annotations

import math
import queue
import threading
import time
from collections import OrderedDict
from concurrent.futures import Future
from dataclasses import dataclass, field

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.bk.config import BKConfig, require_sobol
from nlo_bk_optimized_b200.bk.initial_conditions import MV
from nlo_bk_optimized_b200.dipole.amplitude import BKDipole
from nlo_bk_optimized_b200.dipole.table import DipoleTable
from nlo_bk_optimized_b200.dis.config import Q0sqr, DISConfig


@dataclass(frozen=True)
class Request:
    """One parameter set (MV initial condition) with its DIS points and MC budget."""

    qs0sqr: float
    gamma: float
    ec: float
    points: tuple[tuple[float, float], ...]  # (Q^2, x_Bj)
    budget: int                               # Sobol points per r per stage; Vegas samples follow from it
    seed: int = 0


@dataclass
class Response:
    request: Request
    table: DipoleTable
    F2: torch.Tensor
    FL: torch.Tensor
    FT: torch.Tensor
    sigma_r: torch.Tensor | None
    submitted: float
    finished: float
    cached_table: bool

    @property
    def latency(self) -> float:
        return self.finished - self.submitted


@dataclass
class _Job:
    request: Request
    future: Future
    submitted: float


@dataclass
class ServerStats:
    latencies: list[float] = field(default_factory=list)
    points: int = 0
    requests: int = 0
    cache_hits: int = 0
    started: float = 0.0
    finished: float = 0.0

    def summary(self) -> dict:
        lat = sorted(self.latencies)

        def q(p):
            if not lat:
                return None
            return lat[min(len(lat) - 1, max(0, math.ceil(p * len(lat)) - 1))]

        wall = max(self.finished - self.started, 1e-12)
        return {"requests": self.requests, "points": self.points, "p50_s": q(0.50), "p99_s": q(0.99),
                "points_per_s": self.points / wall, "requests_per_s": self.requests / wall,
                "cache_hits": self.cache_hits, "wall_s": wall}


def dis_options_for(budget: int) -> dict:
    """Vegas settings of a request's DIS integrals from its Monte Carlo budget."""
    return {"vegas_samples": max(4096, budget // 16), "vegas_iterations": 4, "vegas_min_iterations": 4}


def maxy_for(points, margin: float = 0.2, step: float = 0.2) -> float:
    """Evolution range covering every rapidity the request's integrals reach:
    ln(Q^2/(x Q0^2)) of the qqbar-g terms (dis/observables.py:52-54)."""
    need = max(math.log(q2 / (x * Q0sqr)) for q2, x in points)
    return step * math.ceil((need + margin) / step)


class Server:
    def __init__(self, bk_config: BKConfig, dis_config: DISConfig, *, device: torch.device | str = "cuda",
                 slots: int = 8, cache_tables: int = 64, reserve_bytes: int = 1 << 30,
                 sqrt_s: float | None = 318.0):
        require_sobol(bk_config, "the request loop")
        self.bk_config = bk_config
        self.dis_config = dis_config
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the server runs on a CUDA device")
        self.slots = slots
        self.reserve_bytes = reserve_bytes
        self.sqrt_s = sqrt_s
        self.cache: OrderedDict = OrderedDict()
        self.cache_tables = cache_tables
        self._cache_lock = threading.Lock()
        self._queue: queue.Queue = queue.Queue()
        self._free = threading.Semaphore(slots)
        self._stop = threading.Event()
        self.stats = ServerStats()
        self._stats_lock = threading.Lock()
        self._lanes: queue.Queue = queue.Queue()
        lib = _native.load()
        points = bk_config.RPOINTS + 1
        for _ in range(slots):
            self._lanes.put((torch.cuda.Stream(device=self.device),
                             torch.empty(int(lib.nlo_bk_rhs_workspace_bytes(points)), dtype=torch.uint8,
                                         device=self.device)))
        self._scheduler = threading.Thread(target=self._schedule, daemon=True)
        self._scheduler.start()

    # ------------------------------------------------------------------ client side
    def submit(self, request: Request) -> Future:
        future: Future = Future()
        self._queue.put(_Job(request, future, time.perf_counter()))
        return future

    def close(self) -> None:
        self._stop.set()
        self._queue.put(None)
        self._scheduler.join()
        for _ in range(self.slots):  # wait for the running requests
            self._free.acquire()
        torch.cuda.synchronize(self.device)

    # ------------------------------------------------------------------ server side
    def _bytes_needed(self, request: Request) -> int:
        points = self.bk_config.RPOINTS + 1
        steps = int(round(maxy_for(request.points, step=self.bk_config.DE_SOLVER_STEP) / self.bk_config.DE_SOLVER_STEP))
        table = 8 * (steps + 1) * points
        dis = 64 << 20  # Vegas workspaces and states of a request's integrals (generous)
        return table + dis

    def _schedule(self) -> None:
        while True:
            job = self._queue.get()
            if job is None:
                return
            self._free.acquire()  # a slot
            need = self._bytes_needed(job.request)
            for _ in range(1000):  # admission by free device memory
                free, _ = torch.cuda.mem_get_info(self.device)
                if free - need >= self.reserve_bytes:
                    break
                with self._cache_lock:
                    if self.cache:
                        self.cache.popitem(last=False)  # evict the least recently used table
                        continue
                time.sleep(0.005)
            threading.Thread(target=self._run, args=(job,), daemon=True).start()

    def _table(self, request: Request, stream: torch.cuda.Stream, workspace: torch.Tensor) -> tuple[DipoleTable, bool]:
        from nlo_bk_optimized_b200.bk.evolution import _r_grid, _steps_to, nlo_box, params_of, precision_of

        maxy = maxy_for(request.points, step=self.bk_config.DE_SOLVER_STEP)
        key = (request.qs0sqr, request.gamma, request.ec, request.budget, request.seed, maxy)
        with self._cache_lock:
            if key in self.cache:
                self.cache.move_to_end(key)
                return self.cache[key], True
        config = self.bk_config
        lib = _native.load()
        r_host = _r_grid(config, device="cpu", dtype=torch.float64)
        ic = MV(qs0sqr=request.qs0sqr, gamma=request.gamma, ec=request.ec)
        ys = _steps_to(0.0, maxy, config.DE_SOLVER_STEP)
        r = r_host.to(self.device, non_blocking=True)
        rows = torch.empty((len(ys) + 1, r.numel()), dtype=torch.float64, device=self.device)
        rows[0] = ic.dipole_amplitude(r_host).to(torch.float64).to(self.device, non_blocking=True)
        status = torch.zeros(1, dtype=torch.int32, device=self.device)
        lower, width = nlo_box(float(r_host[0]), float(r_host[-1]))
        params = params_of(config, precision_of(config, torch.float32))
        _native.check(lib.nlo_bk_evolve(params, r.data_ptr(), r.numel(), len(ys), float(config.DE_SOLVER_STEP),
                                        _native.STEPPERS[config.stepper], _native.sobol_dirs(4, request.seed),
                                        int(request.budget), _native.box(lower, width), rows.data_ptr(),
                                        status.data_ptr(), workspace.data_ptr(), workspace.numel(),
                                        stream.cuda_stream))
        if int(status.item()) != 0:
            raise FloatingPointError("non-finite BK amplitude")
        y = torch.tensor([0.0, *ys], dtype=torch.float64, device=self.device)
        table = DipoleTable(r=r, y=y, N=rows, x0=ic.x0)
        with self._cache_lock:
            self.cache[key] = table
            while len(self.cache) > self.cache_tables:
                self.cache.popitem(last=False)
        return table, False

    def _run(self, job: _Job) -> None:
        from nlo_bk_optimized_b200.dis.observables import structure_functions

        stream, workspace = self._lanes.get()
        try:
            with torch.cuda.device(self.device), torch.cuda.stream(stream):
                with self._stats_lock:
                    if self.stats.requests == 0 and not self.stats.started:
                        self.stats.started = job.submitted
                table, cached = self._table(job.request, stream, workspace)
                dipole = BKDipole(table)
                Q2 = torch.tensor([p[0] for p in job.request.points], dtype=torch.float64)
                xs = torch.tensor([p[1] for p in job.request.points], dtype=torch.float64)
                sf = structure_functions(Q2, xs, dipole, self.dis_config, sqrt_s=self.sqrt_s, seed=job.request.seed,
                                         **dis_options_for(job.request.budget))
                stream.synchronize()
            done = time.perf_counter()
            response = Response(job.request, table, sf["F2"], sf["FL"], sf["FT"], sf.get("sigma_r"), job.submitted,
                                done, cached)
            with self._stats_lock:
                self.stats.latencies.append(response.latency)
                self.stats.points += len(job.request.points)
                self.stats.requests += 1
                self.stats.cache_hits += int(cached)
                self.stats.finished = max(self.stats.finished, done)
            job.future.set_result(response)
        except BaseException as exc:  # the error goes to the caller's future
            job.future.set_exception(exc)
        finally:
            self._lanes.put((stream, workspace))
            self._free.release()


def run_alone(request: Request, bk_config: BKConfig, dis_config: DISConfig, *, device="cuda",
              sqrt_s: float | None = 318.0) -> Response:
    """The plain path: one request on the default stream, nothing else in flight."""
    server = Server(bk_config, dis_config, device=device, slots=1, cache_tables=0, sqrt_s=sqrt_s)
    try:
        return server.submit(request).result()
    finally:
        server.close()


__all__ = ["Request", "Response", "Server", "ServerStats", "dis_options_for", "maxy_for", "run_alone"]
