"""A request loop for BK tables and DIS structure functions with continuous batching.

A request is one initial-condition parameter set, a list of (Q^2, x_Bj) points and a
Monte Carlo budget.  The server

* admits queued requests while an in-flight slot is free and the device has the memory the
  request needs (evicting least-recently-used resident tables first; a request is never
  admitted past the memory check, and one that cannot fit even on an idle device fails
  with MemoryError);
* evolves each admitted request's table (``nlo_bk_evolve``) on one of several CUDA streams,
  so evolutions of requests that arrived at different times run side by side, and keeps
  evolved N(Y, r) tables resident in an LRU cache keyed by what determines them (parameter
  set, budget, seed, rapidity range);
* runs the DIS integrals of every request whose table is ready in one batch
  (``structure_functions_many``: all points of all those requests, each with its own table
  and seed, in the same few launches per term), on its own stream while the next
  evolutions proceed; requests that become ready during a batch join the next one.

Each request's integrals are the same computation as when it runs alone; only the CTA
partition of the merged launches (and so the order of FP64 partial sums) differs, which the
adaptive grids carry to ~1e-9 relative.  Latency is measured per request from ``submit`` to
completion; ``stats`` reports p50/p99 and the point throughput.
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
    """Vegas settings of a request's DIS integrals from its Monte Carlo budget: 4 iterations of
    the power of two nearest budget/16 samples (at least 4096), so that requests of similar
    budgets share the merged launches."""
    samples = max(4096, 1 << max(0, round(math.log2(max(budget, 1) / 16))))
    return {"vegas_samples": samples, "vegas_iterations": 4, "vegas_min_iterations": 4}


def maxy_for(points, margin: float = 0.2, step: float = 0.2) -> float:
    """Evolution range covering every rapidity the request's integrals reach:
    ln(Q^2/(x Q0^2)) of the qqbar-g terms (dis/observables.py:52-54)."""
    need = max(math.log(q2 / (x * Q0sqr)) for q2, x in points)
    return step * math.ceil((need + margin) / step)


def request_table(request: Request, config: BKConfig, device: torch.device, stream: torch.cuda.Stream,
                  workspace: torch.Tensor) -> DipoleTable:
    """The request's N(Y, r) table: its MV initial condition evolved with ``nlo_bk_evolve`` on
    `stream` to the rapidity its points need, with its budget and seed."""
    from nlo_bk_optimized_b200.bk.evolution import _r_grid, _steps_to, nlo_box, params_of, precision_of

    maxy = maxy_for(request.points, step=config.DE_SOLVER_STEP)
    lib = _native.load()
    r_host = _r_grid(config, device="cpu", dtype=torch.float64)
    ic = MV(qs0sqr=request.qs0sqr, gamma=request.gamma, ec=request.ec)
    ys = _steps_to(0.0, maxy, config.DE_SOLVER_STEP)
    r = r_host.to(device, non_blocking=True)
    rows = torch.empty((len(ys) + 1, r.numel()), dtype=torch.float64, device=device)
    rows[0] = ic.dipole_amplitude(r_host).to(torch.float64).to(device, non_blocking=True)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    lower, width = nlo_box(float(r_host[0]), float(r_host[-1]))
    params = params_of(config, precision_of(config, torch.float32))
    _native.check(lib.nlo_bk_evolve(params, r.data_ptr(), r.numel(), len(ys), float(config.DE_SOLVER_STEP),
                                    _native.STEPPERS[config.stepper], _native.sobol_dirs(4, request.seed),
                                    int(request.budget), _native.box(lower, width), rows.data_ptr(),
                                    status.data_ptr(), workspace.data_ptr(), workspace.numel(), stream.cuda_stream))
    if int(status.item()) != 0:
        raise FloatingPointError("non-finite BK amplitude")
    y = torch.tensor([0.0, *ys], dtype=torch.float64, device=device)
    return DipoleTable(r=r, y=y, N=rows, x0=ic.x0)


@dataclass
class _Ready:
    job: _Job
    table: DipoleTable
    dipole: BKDipole
    cached: bool


class Server:
    def __init__(self, bk_config: BKConfig, dis_config: DISConfig, *, device: torch.device | str = "cuda",
                 slots: int = 64, lanes: int = 8, cache_tables: int = 64, reserve_bytes: int = 1 << 30,
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
        self._inflight = 0
        self._inflight_lock = threading.Lock()
        self._ready: list[_Ready] = []
        self._ready_cv = threading.Condition()
        self._stop = threading.Event()
        self.stats = ServerStats()
        self._stats_lock = threading.Lock()
        self.batches: list[int] = []  # requests per DIS batch
        lib = _native.load()
        points = bk_config.RPOINTS + 1
        self._lanes: queue.Queue = queue.Queue()
        for _ in range(max(1, lanes)):
            self._lanes.put((torch.cuda.Stream(device=self.device),
                             torch.empty(int(lib.nlo_bk_rhs_workspace_bytes(points)), dtype=torch.uint8,
                                         device=self.device)))
        self._dis_stream = torch.cuda.Stream(device=self.device)
        self._scheduler = threading.Thread(target=self._schedule, daemon=True)
        self._batcher = threading.Thread(target=self._dis_loop, daemon=True)
        self._scheduler.start()
        self._batcher.start()

    # ------------------------------------------------------------------ client side
    def submit(self, request: Request) -> Future:
        future: Future = Future()
        self._queue.put(_Job(request, future, time.perf_counter()))
        return future

    def close(self) -> None:
        self._queue.put(None)
        self._scheduler.join()
        for _ in range(self.slots):  # every admitted request has finished
            self._free.acquire()
        self._stop.set()
        with self._ready_cv:
            self._ready_cv.notify_all()
        self._batcher.join()
        torch.cuda.synchronize(self.device)

    # ------------------------------------------------------------------ server side
    def _bytes_needed(self, request: Request) -> int:
        points = self.bk_config.RPOINTS + 1
        steps = int(round(maxy_for(request.points, step=self.bk_config.DE_SOLVER_STEP) / self.bk_config.DE_SOLVER_STEP))
        table = 8 * (steps + 1) * points
        dis = (4 << 20) * max(1, len(request.points))  # the request's share of a merged DIS batch
        return table + dis

    def _finish(self, job: _Job, exc: BaseException | None = None, response: Response | None = None) -> None:
        if exc is not None:
            job.future.set_exception(exc)
        else:
            job.future.set_result(response)
        with self._inflight_lock:
            self._inflight -= 1
        self._free.release()

    def _schedule(self) -> None:
        total = torch.cuda.get_device_properties(self.device).total_memory
        while True:
            job = self._queue.get()
            if job is None:
                return
            self._free.acquire()  # an in-flight slot
            with self._inflight_lock:
                self._inflight += 1
            with self._stats_lock:
                if not self.stats.started:
                    self.stats.started = job.submitted
            need = self._bytes_needed(job.request)
            if need + self.reserve_bytes > total:
                self._finish(job, MemoryError(f"a request needing {need} bytes cannot fit on the device"))
                continue
            while True:  # admission by free device memory: wait, evicting resident tables first
                free, _ = torch.cuda.mem_get_info(self.device)
                if free - need >= self.reserve_bytes:
                    break
                with self._cache_lock:
                    if self.cache:
                        self.cache.popitem(last=False)  # the least recently used table
                        torch.cuda.empty_cache()
                        continue
                time.sleep(0.005)
            threading.Thread(target=self._evolve, args=(job,), daemon=True).start()

    def _table(self, request: Request, stream: torch.cuda.Stream, workspace: torch.Tensor) -> tuple[DipoleTable, bool]:
        maxy = maxy_for(request.points, step=self.bk_config.DE_SOLVER_STEP)
        key = (request.qs0sqr, request.gamma, request.ec, request.budget, request.seed, maxy)
        with self._cache_lock:
            if key in self.cache:
                self.cache.move_to_end(key)
                return self.cache[key], True
        table = request_table(request, self.bk_config, self.device, stream, workspace)
        with self._cache_lock:
            self.cache[key] = table
            while len(self.cache) > self.cache_tables:
                self.cache.popitem(last=False)
        return table, False

    def _evolve(self, job: _Job) -> None:
        stream, workspace = self._lanes.get()
        try:
            with torch.cuda.device(self.device), torch.cuda.stream(stream):
                table, cached = self._table(job.request, stream, workspace)
                dipole = BKDipole(table)
                stream.synchronize()
            with self._ready_cv:
                self._ready.append(_Ready(job, table, dipole, cached))
                self._ready_cv.notify()
        except BaseException as exc:  # the error goes to the caller's future
            self._finish(job, exc)
        finally:
            self._lanes.put((stream, workspace))

    def _dis_loop(self) -> None:
        from nlo_bk_optimized_b200.dis.observables import structure_functions_many

        while True:
            with self._ready_cv:
                while not self._ready and not self._stop.is_set():
                    self._ready_cv.wait(timeout=0.05)
                if not self._ready and self._stop.is_set():
                    return
                batch, self._ready = self._ready, []
            self.batches.append(len(batch))
            Q2, xs, dipoles, seeds, options, owner = [], [], [], [], [], []
            for k, item in enumerate(batch):
                opts = dis_options_for(item.job.request.budget)
                for q2, x in item.job.request.points:
                    Q2.append(q2)
                    xs.append(x)
                    dipoles.append(item.dipole)
                    seeds.append(item.job.request.seed)
                    options.append(opts)
                    owner.append(k)
            try:
                with torch.cuda.device(self.device), torch.cuda.stream(self._dis_stream):
                    sf = structure_functions_many(Q2, xs, dipoles, self.dis_config, sqrt_s=self.sqrt_s, seeds=seeds,
                                                  options=options)
                    sf = {k: v.cpu() for k, v in sf.items()}
            except BaseException as exc:
                for item in batch:
                    self._finish(item.job, exc)
                continue
            done = time.perf_counter()
            owner_t = torch.tensor(owner)
            for k, item in enumerate(batch):
                sel = owner_t == k
                response = Response(item.job.request, item.table, sf["F2"][sel], sf["FL"][sel], sf["FT"][sel],
                                    sf["sigma_r"][sel] if "sigma_r" in sf else None, item.job.submitted, done,
                                    item.cached)
                with self._stats_lock:
                    self.stats.latencies.append(response.latency)
                    self.stats.points += len(item.job.request.points)
                    self.stats.requests += 1
                    self.stats.cache_hits += int(item.cached)
                    self.stats.finished = max(self.stats.finished, done)
                self._finish(item.job, response=response)


def run_alone(request: Request, bk_config: BKConfig, dis_config: DISConfig, *, device="cuda",
              sqrt_s: float | None = 318.0) -> Response:
    """The plain single-solve path: the request's evolution and then its points' structure
    functions (``structure_functions``), on the current stream, nothing else in flight."""
    from nlo_bk_optimized_b200.dis.observables import structure_functions

    require_sobol(bk_config, "the request loop")
    device = torch.device(device)
    submitted = time.perf_counter()
    lib = _native.load()
    workspace = torch.empty(int(lib.nlo_bk_rhs_workspace_bytes(bk_config.RPOINTS + 1)), dtype=torch.uint8,
                            device=device)
    table = request_table(request, bk_config, device, torch.cuda.current_stream(device), workspace)
    dipole = BKDipole(table)
    Q2 = torch.tensor([p[0] for p in request.points], dtype=torch.float64)
    xs = torch.tensor([p[1] for p in request.points], dtype=torch.float64)
    sf = structure_functions(Q2, xs, dipole, dis_config, sqrt_s=sqrt_s, seed=request.seed,
                             **dis_options_for(request.budget))
    sf = {k: v.cpu() for k, v in sf.items()}
    return Response(request, table, sf["F2"], sf["FL"], sf["FT"], sf.get("sigma_r"), submitted, time.perf_counter(),
                    False)


__all__ = ["Request", "Response", "Server", "ServerStats", "dis_options_for", "maxy_for", "request_table",
           "run_alone"]
