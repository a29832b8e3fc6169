"""A request loop for BK tables and DIS structure functions with continuous batching.

A request is one initial-condition parameter set, a list of (Q^2, x_Bj) points and a
Monte Carlo budget.  The server

* admits queued requests while an in-flight slot is free and the device has the memory the
  request needs (evicting least-recently-used resident tables first; a request is never
  admitted past the memory check, and one that cannot fit even on an idle device fails
  with MemoryError);
* batches the BK evolutions at the level of rapidity steps: one engine thread advances every
  in-flight evolution by one step per ``nlo_bk_evolve_sets`` call (one launch per kernel and
  stage for all of them, each with its own initial row, budget and seed); a request admitted
  while others are evolving joins at the next step, and one that reaches its rapidity leaves
  -- the iteration-level batching of a decode loop, applied to the rapidity steps;
* keeps evolved N(Y, r) tables resident in an LRU cache keyed by what determines them
  (parameter set, budget, seed, rapidity range); a request whose table is resident or being
  evolved for an earlier request takes that table;
* runs the DIS integrals of every request whose table is ready in one batch
  (``structure_functions_many``: all points of all those requests, each with its own table
  and seed, in the same few launches per term), on its own stream while the next rapidity
  steps proceed; requests that become ready during a batch join the next one.

Each request's results are the same computation as when it runs alone: its table equals its
own evolution up to the order of the FP64 sums of the multi-set launches' CTA partials
(~1e-15), and its integrals differ only by the CTA partition of the merged launches, which
the adaptive grids carry to ~1e-9 relative.  Latency is measured per request from ``submit``
to completion; ``stats`` reports p50/p99 and the point throughput.
"""

from __future__ import annotations

import ctypes
import math
import queue
import threading
import time
from collections import OrderedDict
from concurrent.futures import Future
from dataclasses import dataclass, field

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.bk.batch import DEFAULT_WAVES, MAX_SETS
from nlo_bk_optimized_b200.bk.config import BKConfig, require_fixed_step, require_sobol
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
    cached: bool
    done: torch.cuda.Event | None  # recorded after the table's last rapidity step


@dataclass
class _Flight:
    """An evolution in progress: rows [steps+1, R], row `step` the current amplitude."""

    key: tuple
    jobs: list
    rows: torch.Tensor
    y: torch.Tensor
    x0: float
    steps: int
    budget: int
    dirs: object
    step: int = 0


class Server:
    def __init__(self, bk_config: BKConfig, dis_config: DISConfig, *, device: torch.device | str = "cuda",
                 slots: int = 64, waves: int = DEFAULT_WAVES, cache_tables: int = 64, reserve_bytes: int = 1 << 30,
                 sqrt_s: float | None = 318.0):
        from nlo_bk_optimized_b200.bk.evolution import _r_grid, nlo_box, params_of, precision_of

        require_sobol(bk_config, "the request loop")
        require_fixed_step(bk_config, "the request loop")
        if bk_config.KINEMATICAL_CONSTRAINT:
            raise NotImplementedError("the request loop evolves without the kinematical constraint")
        self.bk_config = bk_config
        self.dis_config = dis_config
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the server runs on a CUDA device")
        self.slots = slots
        self.waves = waves
        self.reserve_bytes = reserve_bytes
        self.sqrt_s = sqrt_s
        self.cache: OrderedDict = OrderedDict()
        self.cache_tables = cache_tables
        self._cache_lock = threading.Lock()
        self._queue: queue.Queue = queue.Queue()    # submitted jobs
        self._joining: queue.Queue = queue.Queue()  # admitted jobs for the engine
        self._free = threading.Semaphore(slots)
        self._inflight = 0
        self._inflight_lock = threading.Lock()
        self._ready: list[_Ready] = []
        self._ready_cv = threading.Condition()
        self._stop = threading.Event()
        self.stats = ServerStats()
        self._stats_lock = threading.Lock()
        self.batches: list[int] = []     # requests per DIS batch
        self.step_sets: list[int] = []  # evolutions advanced per engine step
        lib = _native.load()
        r_host = _r_grid(bk_config, device="cpu", dtype=torch.float64)
        self._r_host = r_host
        self._r = r_host.to(self.device)
        self._points = r_host.numel()
        lower, width = nlo_box(float(r_host[0]), float(r_host[-1]))
        self._box = _native.box(lower, width)
        self._params = params_of(bk_config, precision_of(bk_config, torch.float32))
        self._per_call = max(1, min(slots, MAX_SETS))
        ws = max(int(lib.nlo_bk_sets_workspace_bytes(self._points, n, waves)) for n in range(1, self._per_call + 1))
        self._workspace = torch.empty(ws, dtype=torch.uint8, device=self.device)
        self._status = torch.zeros(self._per_call, dtype=torch.int32, device=self.device)
        self._bk_stream = torch.cuda.Stream(device=self.device)
        self._dis_stream = torch.cuda.Stream(device=self.device)
        self._scheduler = threading.Thread(target=self._schedule, daemon=True)
        self._engine = threading.Thread(target=self._bk_loop, daemon=True)
        self._batcher = threading.Thread(target=self._dis_loop, daemon=True)
        self._scheduler.start()
        self._engine.start()
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
        self._engine.join()
        with self._ready_cv:
            self._ready_cv.notify_all()
        self._batcher.join()
        torch.cuda.synchronize(self.device)

    # ------------------------------------------------------------------ server side
    def _bytes_needed(self, request: Request) -> int:
        steps = int(round(maxy_for(request.points, step=self.bk_config.DE_SOLVER_STEP) / self.bk_config.DE_SOLVER_STEP))
        table = 8 * (steps + 1) * self._points
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
            self._joining.put(job)

    def _key(self, request: Request) -> tuple:
        maxy = maxy_for(request.points, step=self.bk_config.DE_SOLVER_STEP)
        return (request.qs0sqr, request.gamma, request.ec, request.budget, request.seed, maxy)

    def _ready_add(self, item: _Ready) -> None:
        with self._ready_cv:
            self._ready.append(item)
            self._ready_cv.notify()

    def _join(self, job: _Job, flights: list[_Flight]) -> None:
        """A newly admitted request: a resident table, a table already being evolved, or a new
        evolution starting at the next step."""
        from nlo_bk_optimized_b200.bk.evolution import _steps_to

        request = job.request
        key = self._key(request)
        with self._cache_lock:
            if key in self.cache:
                self.cache.move_to_end(key)
                table, done = self.cache[key]
                self._ready_add(_Ready(job, table, True, done))
                return
        for flight in flights:
            if flight.key == key:
                flight.jobs.append(job)
                return
        ys = _steps_to(0.0, key[-1], self.bk_config.DE_SOLVER_STEP)
        ic = MV(qs0sqr=request.qs0sqr, gamma=request.gamma, ec=request.ec)
        rows = torch.empty((len(ys) + 1, self._points), dtype=torch.float64, device=self.device)
        rows[0] = ic.dipole_amplitude(self._r_host).to(torch.float64).to(self.device)
        y = torch.tensor([0.0, *ys], dtype=torch.float64, device=self.device)
        flights.append(_Flight(key, [job], rows, y, ic.x0, len(ys), int(request.budget),
                               _native.sobol_dirs(4, request.seed)))

    def _step(self, flights: list[_Flight]) -> None:
        """One rapidity step of every flight (at most MAX_SETS per call) on the engine stream."""
        lib = _native.load()
        R = self._points
        for start in range(0, len(flights), self._per_call):
            chunk = flights[start:start + self._per_call]
            n = len(chunk)
            ptrs = (ctypes.c_void_p * n)(*[f.rows.data_ptr() + 8 * R * f.step for f in chunk])
            budgets = (ctypes.c_int64 * n)(*[f.budget for f in chunk])
            dirs = (_native.SobolDirs * n)(*[f.dirs for f in chunk])
            _native.check(lib.nlo_bk_evolve_sets(self._params, self._r.data_ptr(), R, n, ptrs, 1,
                                                 float(self.bk_config.DE_SOLVER_STEP),
                                                 _native.STEPPERS[self.bk_config.stepper], dirs, budgets, self._box,
                                                 self.waves, self._status.data_ptr(), self._workspace.data_ptr(),
                                                 self._workspace.numel(), self._bk_stream.cuda_stream))
        for f in flights:
            f.step += 1

    def _bk_loop(self) -> None:
        flights: list[_Flight] = []
        previous: torch.cuda.Event | None = None
        with torch.cuda.device(self.device):
            while True:
                # admitted requests join before the next step (wait only while nothing evolves)
                while True:
                    try:
                        job = self._joining.get(block=not flights, timeout=0.02)
                    except queue.Empty:
                        break
                    try:
                        with torch.cuda.stream(self._bk_stream):
                            self._join(job, flights)
                    except BaseException as exc:  # the error goes to the caller's future
                        self._finish(job, exc)
                if not flights:
                    if self._stop.is_set() and self._joining.empty():
                        return
                    continue
                try:
                    self._step(flights)
                except BaseException as exc:
                    for f in flights:
                        for job in f.jobs:
                            self._finish(job, exc)
                    flights = []
                    continue
                self.step_sets.append(len(flights))
                done = torch.cuda.Event()
                done.record(self._bk_stream)
                for f in [f for f in flights if f.step == f.steps]:
                    table = DipoleTable(r=self._r, y=f.y, N=f.rows, x0=f.x0)
                    with self._cache_lock:
                        self.cache[f.key] = (table, done)
                        while len(self.cache) > self.cache_tables:
                            self.cache.popitem(last=False)
                    for k, job in enumerate(f.jobs):
                        self._ready_add(_Ready(job, table, k > 0, done))
                flights = [f for f in flights if f.step < f.steps]
                # keep at most two steps queued: new requests join within a step
                if previous is not None:
                    previous.synchronize()
                previous = done

    def _dis_loop(self) -> None:
        from nlo_bk_optimized_b200.dis.observables import structure_functions_many

        while True:
            with self._ready_cv:
                while not self._ready and not self._stop.is_set():
                    self._ready_cv.wait(timeout=0.05)
                if not self._ready and self._stop.is_set():
                    return
                batch, self._ready = self._ready, []
            good = []
            with torch.cuda.device(self.device), torch.cuda.stream(self._dis_stream):
                for item in batch:
                    if item.done is not None:
                        item.done.synchronize()
                    if not bool(torch.isfinite(item.table.N).all()):
                        self._finish(item.job, FloatingPointError("non-finite BK amplitude"))
                    else:
                        good.append(item)
            batch = good
            if not batch:
                continue
            self.batches.append(len(batch))
            Q2, xs, dipoles, seeds, options, owner = [], [], [], [], [], []
            for k, item in enumerate(batch):
                opts = dis_options_for(item.job.request.budget)
                # the table was written on the engine stream: keep its memory until this stream is done
                item.table.N.record_stream(self._dis_stream)
                item.table.y.record_stream(self._dis_stream)
                dipole = BKDipole(item.table)
                for q2, x in item.job.request.points:
                    Q2.append(q2)
                    xs.append(x)
                    dipoles.append(dipole)
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
    require_fixed_step(bk_config, "the request loop")
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
