"""NLO DIS cross sections and structure functions on the device (interface of the
reference's dis/observables.py:1-742 and dis/lo.py).

Every integral is one "job" of libnlo_b200.so: the LO term and the 2D virtual term by
the tensor Gauss-Legendre rule (``nlo_dis_gauss_legendre``), the 3D/4D virtual terms and
the qqbar-g terms by the device Vegas (``nlo_dis_vegas``).  Jobs of one term -- all
quarks, polarisations and kinematic points of a request -- run in the same launches, and
the host reads the results once.  The single-point functions (``F2``, ``FL``, ``FT``,
``photon_proton_cross_section_d2b`` ...) keep the reference's signatures, seeds and
budget rules and run through the same batched engine with one point;
``structure_functions`` takes many points at once.

Vegas samples are the scrambled Sobol points of SobolEngine(dims, scramble=True, seed)
split into a bin and a fraction per dimension, where the reference draws torch.randint
bins and torch.rand fractions from a generator with the same seed.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import torch

from nlo_bk_optimized_b200 import _native
from nlo_bk_optimized_b200.dipole.amplitude import GBW, BKDipole
from nlo_bk_optimized_b200.dis.config import (
    NC,
    AlphaEM,
    DISConfig,
    DISOrder,
    HeavyQuarkX,
    NcScheme,
    Polarization,
    Q0sqr,
    Quark,
    RunningCouplingIRScheme,
    RunningCouplingScheme,
)
from nlo_bk_optimized_b200.numerics.integration import (
    IntegralResult,
    VegasOptions,
    budget_options,
    gauss_legendre_terms,
    state_results,
    vegas_terms,
)

ZMIN = 1e-6
Dipole = GBW | BKDipole
TERMS = _native.DIS_TERMS
LO_FACTOR = 4 * AlphaEM * NC / (2 * math.pi) ** 2
DIP_FACTOR = 4 * NC * AlphaEM / (2 * math.pi) ** 2 * 2 * math.pi
QG_FACTOR = 4 * NC * AlphaEM / (2 * math.pi) ** 3 * 2 * math.pi
_DIP_CONTRIBUTIONS = {Polarization.T: ("T0", "T1", "T2"), Polarization.L: ("Omega_L_const", "ab", "cd")}


# ----------------------------------------------------------------------------- helpers


def _precision(config: DISConfig, reference: torch.Tensor | None = None) -> int:
    if config.precision == "fp64":
        return _native.PRECISION_FP64
    return _native.PRECISION_MIXED


def _device(*tensors) -> torch.device:
    for t in tensors:
        if isinstance(t, torch.Tensor) and t.is_cuda:
            return t.device
    if not torch.cuda.is_available():
        raise RuntimeError("the DIS path runs on CUDA devices only (no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def kinematics(Q2: float, xbj: float, polarization: Polarization, config: DISConfig,
               quark: Quark | None = None) -> _native.DisKinematics:
    """The job description of one (Q^2, x_Bj, polarisation[, quark]) for the C ABI."""
    k = _native.DisKinematics()
    k.Q2 = float(Q2)
    k.xbj = float(xbj)
    k.mf = float(quark.mass) if quark is not None else 0.0
    k.n_quarks = len(config.quarks)
    for i, q in enumerate(config.quarks):
        k.lo_mass[i] = q.mass
        k.lo_charge2[i] = q.charge**2
    k.maxr = config.maxr
    k.transverse = int(polarization is Polarization.T)
    k.finite_nc = int(config.nc_scheme is NcScheme.FiniteNC)
    k.parent_coupling = int(config.rc_scheme is RunningCouplingScheme.PARENT)
    k.smooth_coupling = int(config.rc_ir_scheme is RunningCouplingIRScheme.SMOOTH)
    k.mass_dependent_x = int(config.heavy_quark_x_scheme is HeavyQuarkX.MassDependentX)
    k.c2_alpha = config.C2_alpha
    k.active_flavors = float(config.active_flavors)
    k.max_alpha = config.max_alpha_s_freeze
    return k


def _validate_kinematics(Q2: torch.Tensor, xbj: torch.Tensor) -> None:
    if Q2.numel() != 1 or xbj.numel() != 1:
        raise ValueError("Q2 and xbj must be scalar tensors")
    if Q2.device != xbj.device or Q2.dtype != xbj.dtype:
        raise ValueError("Q2 and xbj must have the same device and dtype")
    if not bool(torch.isfinite(Q2)) or not bool(torch.isfinite(xbj)):
        raise ValueError("Q2 and xbj must be finite")
    if not bool(Q2 > 0) or not bool((xbj > 0) & (xbj <= 1)):
        raise ValueError("Q2 must be positive and xbj must lie in (0, 1]")


def _scale_result(result: IntegralResult, factor: float) -> IntegralResult:
    return IntegralResult(result.value * factor, result.error * abs(factor), result.n_eval, result.converged,
                          result.seed)


def _sum_results(results, seed: int | None) -> IntegralResult:
    if not results:
        raise ValueError("at least one integration result is required")
    value = torch.stack([r.value for r in results]).sum()
    error = torch.sqrt(torch.stack([r.error.square() for r in results]).sum())
    return IntegralResult(value, error, sum(r.n_eval for r in results), all(r.converged for r in results), seed)


def dipole_rapidity(Q2: float, xbj: float, mf: float, scheme: HeavyQuarkX) -> float:
    W2 = (1 - xbj) * Q2 / xbj
    X = (Q2 + 4 * mf**2) / (Q2 + W2) if scheme is HeavyQuarkX.MassDependentX else Q2 / (Q2 + W2)
    return math.log(1 / X)


# ----------------------------------------------------------------------------- the job engine


@dataclass
class _Job:
    term: int
    kin: _native.DisKinematics
    seed: int = 0
    options: VegasOptions | None = None  # None: tensor Gauss-Legendre
    points: int = 24
    lo_Y: float | None = None            # LO jobs on a BK table: rapidity to initialise at
    fixed: tuple | None = None           # fixed-Sobol qqbar-g job: (polarisation, quark)
    dipole: Dipole | None = None         # None: the engine's dipole
    done: bool = False
    value: float = 0.0
    error: float = 0.0
    n_eval: int = 0
    converged: bool = False


@dataclass
class _Engine:
    dipole: Dipole
    config: DISConfig
    device: torch.device
    jobs: list[_Job] = field(default_factory=list)

    def add(self, job: _Job) -> _Job:
        if job.dipole is None:
            job.dipole = self.dipole
        self.jobs.append(job)
        return job

    @staticmethod
    def _natives(group: list[_Job]):
        """One native dipole for a group on one dipole, else one per job."""
        first = group[0].dipole
        if all(j.dipole is first for j in group):
            return first.native(), None
        return None, [j.dipole.native() for j in group]

    def run(self) -> None:
        precision = _precision(self.config)
        pending = []
        todo = [j for j in self.jobs if not j.done]
        for job in todo:
            if job.fixed is not None:
                from nlo_bk_optimized_b200.dis.fixed_sobol import FIXED_SOBOL_EVALUATIONS, fixed_sobol_device

                pol, quark = job.fixed
                _, est = fixed_sobol_device(job.kin.Q2, job.kin.xbj, pol, quark, job.dipole, self.config,
                                            seed=job.seed, device=self.device, precision=precision)
                pending.append(("fixed", [job], est))
        todo = [j for j in todo if j.fixed is None]
        # Gauss-Legendre jobs first, grouped by the table rapidity they initialise at (the
        # reference initialises the BK table before each LO integral, and the later terms
        # see that state)
        gl_groups: dict[tuple, list[_Job]] = {}
        for job in todo:
            if job.options is None:
                gl_groups.setdefault((job.lo_Y if job.term == TERMS["LO"] else None, job.term, job.points),
                                     []).append(job)
        # LO groups first (each after initialising the table at its rapidity), then the
        # other Gauss-Legendre terms, then Vegas: the order of photon_proton_cross_section_d2b
        order = sorted(gl_groups, key=lambda key: (key[0] is None, key[0] or 0.0))
        for key in order:
            lo_Y, term, points = key
            group = gl_groups[key]
            if lo_Y is not None:
                tables = {id(j.dipole): j.dipole for j in group if isinstance(j.dipole, BKDipole)}
                for table in tables.values():
                    table.initialize_interpolation(lo_Y)
            native, natives = self._natives(group)
            out = gauss_legendre_terms(term, [j.kin for j in group], native, points, precision=precision,
                                       device=self.device, dipoles=natives)
            pending.append(("gl", group, out))
        vegas_groups: dict[tuple, list[_Job]] = {}
        for job in todo:
            if job.options is not None:
                vegas_groups.setdefault((job.term, job.options), []).append(job)
        for (term, options), group in vegas_groups.items():
            native, natives = self._natives(group)
            state = vegas_terms(term, [j.kin for j in group], native, options, [j.seed for j in group],
                                precision=precision, device=self.device, dipoles=natives)
            pending.append(("vegas", group, state_results(state, term, options.bins)))
        for kind, group, out in pending:
            for job in group:
                job.done = True
            if kind == "fixed":
                est = out.cpu()
                job = group[0]
                totals = est.sum(dim=1)
                job.value = float(totals.mean())
                job.error = float(totals.std(unbiased=True) / math.sqrt(totals.numel()))
                job.n_eval = FIXED_SOBOL_EVALUATIONS
                job.converged = job.error <= self.config.epsrel * abs(job.value)
            elif kind == "gl":
                host = out.cpu()
                for j, job in enumerate(group):
                    job.value = float(host[j, 0])
                    job.error = float(host[j, 1])
                    n = job.points
                    job.n_eval = n * n + max(2, n // 2) ** 2
                    job.converged = job.error <= self.config.epsrel * abs(job.value)
            else:
                value, error = out["value"].cpu(), out["error"].cpu()
                evals, conv = out["n_eval"].cpu(), out["converged"].cpu()
                for j, job in enumerate(group):
                    job.value = float(value[j])
                    job.error = float(error[j])
                    job.n_eval = int(evals[j])
                    job.converged = bool(conv[j] != 0)


def _result(job: _Job, scale: float, device: torch.device, seed) -> IntegralResult:
    return IntegralResult(torch.tensor(job.value * scale, dtype=torch.float64, device=device),
                          torch.tensor(job.error * abs(scale), dtype=torch.float64, device=device),
                          job.n_eval, job.converged, seed)


def _lo_Y(dipole: Dipole, xbj: float) -> float:
    return max(math.log(dipole.X0() / xbj), 0.0)


@dataclass
class _SigmaPlan:
    """Jobs of photon_proton_cross_section_d2b for one point and polarisation."""

    lo: _Job
    dip: list[list[_Job]]
    qg: list[list[_Job]]
    seed: int
    qg_fixed: list[_Job] = field(default_factory=list)
    dipole: Dipole | None = None
    Q2: float = 0.0
    xbj: float = 0.0
    pol: Polarization = Polarization.T
    overrides: dict = field(default_factory=dict)


def fixed_sobol_supported(dipole: Dipole, config: DISConfig, single_precision: bool) -> bool:
    """_fixed_sobol_supported (dis/observables.py:644-660): GBW, nested 48-node inner rule,
    a budget of at least FIXED_SOBOL_EVALUATIONS, and the single-precision (mixed) path."""
    from nlo_bk_optimized_b200.dis.fixed_sobol import FIXED_SOBOL_EVALUATIONS

    return (single_precision and config.cuda_fusion and config.cuda_nested and config.cuda_nested_points == 48
            and isinstance(dipole, GBW) and config.maxeval >= FIXED_SOBOL_EVALUATIONS)


def _plan_qg_vegas(engine: "_Engine", plan: _SigmaPlan) -> None:
    config = engine.config
    qg, offset = [], 0
    qg_seed = plan.seed + 100
    nested = config.cuda_nested
    for quark in config.quarks:
        kin = kinematics(plan.Q2, plan.xbj, plan.pol, config, quark)
        opts = _vegas_options(config, config.maxeval, plan.overrides)
        jobs = []
        for term in ("I1", "I2N" if nested else "I2", "I3N" if nested else "I3"):
            jobs.append(engine.add(_Job(TERMS[term], kin, seed=qg_seed + offset, options=opts, dipole=plan.dipole)))
            offset += 1
        qg.append(jobs)
    plan.qg = qg


def _integration_overrides(options: dict) -> dict:
    return {k: options[k] for k in ("vegas_samples", "vegas_iterations", "vegas_bins", "vegas_min_iterations")
            if k in options and options[k] is not None}


def _vegas_options(config: DISConfig, maxeval: int, overrides: dict) -> VegasOptions:
    bins = overrides.get("vegas_bins", config.vegas_bins)
    if "vegas_samples" in overrides or "vegas_iterations" in overrides:
        base = budget_options(maxeval, config.epsrel, bins)
        iterations = overrides.get("vegas_iterations", base.max_iterations)
        return VegasOptions(samples_per_iteration=overrides.get("vegas_samples", base.samples_per_iteration),
                            max_iterations=iterations,
                            min_iterations=min(overrides.get("vegas_min_iterations", base.min_iterations), iterations),
                            bins=bins, epsrel=config.epsrel, inner_points=config.cuda_nested_points)
    base = budget_options(maxeval, config.epsrel, bins)
    return VegasOptions(samples_per_iteration=base.samples_per_iteration, max_iterations=base.max_iterations,
                        min_iterations=base.min_iterations, bins=bins, epsrel=config.epsrel,
                        inner_points=config.cuda_nested_points)


def _plan_lo(engine: _Engine, Q2: float, xbj: float, pol: Polarization, points: int,
             dipole: Dipole | None = None) -> _Job:
    dipole = dipole if dipole is not None else engine.dipole
    kin = kinematics(Q2, xbj, pol, engine.config)
    return engine.add(_Job(TERMS["LO"], kin, points=points, lo_Y=_lo_Y(dipole, xbj), dipole=dipole))


def _plan_sigma(engine: _Engine, Q2: float, xbj: float, pol: Polarization, *, seed: int, points: int,
                overrides: dict, fixed: bool = False, dipole: Dipole | None = None) -> _SigmaPlan:
    config = engine.config
    dipole = dipole if dipole is not None else engine.dipole
    if config.order is DISOrder.LO:
        return _SigmaPlan(_plan_lo(engine, Q2, xbj, pol, points, dipole), [], [], seed, dipole=dipole)
    lo = _plan_lo(engine, Q2, dipole.X0(), pol, points, dipole)
    if isinstance(dipole, BKDipole):
        Ymax = max(dipole_rapidity(Q2, xbj, q.mass, config.heavy_quark_x_scheme) for q in config.quarks)
        dipole.check_rapidity(max(Ymax, math.log(Q2 / xbj / Q0sqr)))
    dip, offset = [], 0
    for quark in config.quarks:
        kin = kinematics(Q2, xbj, pol, config, quark)
        opts = _vegas_options(config, config.maxeval * (10 if quark.mass < 0.4 else 1), overrides)
        jobs = [engine.add(_Job(TERMS["DIP0"], kin, points=points, dipole=dipole))]
        for term in ("DIP1", "DIP2"):
            jobs.append(engine.add(_Job(TERMS[term], kin, seed=seed + offset, options=opts, dipole=dipole)))
            offset += 1
        dip.append(jobs)
    plan = _SigmaPlan(lo, dip, [], seed, dipole=dipole, Q2=Q2, xbj=xbj, pol=pol, overrides=overrides)
    if fixed and fixed_sobol_supported(dipole, config, True):
        for index, quark in enumerate(config.quarks):
            kin = kinematics(Q2, xbj, pol, config, quark)
            plan.qg_fixed.append(engine.add(_Job(-1, kin, seed=seed + 100 + index, fixed=(pol, quark),
                                                 dipole=dipole)))
    else:
        _plan_qg_vegas(engine, plan)
    return plan


def _run_with_fallback(engine: _Engine, plans: list[_SigmaPlan]) -> None:
    """Run the engine; where a fixed-Sobol qqbar-g result did not converge, integrate that
    plan's qqbar-g terms by Vegas instead (dis/observables.py:470-489)."""
    engine.run()
    retry = [p for p in plans if p.qg_fixed and not all(j.converged for j in p.qg_fixed)]
    for plan in retry:
        plan.qg_fixed = []
        _plan_qg_vegas(engine, plan)
    if retry:
        engine.run()


def _sigma_result(plan: _SigmaPlan, config: DISConfig, device: torch.device) -> IntegralResult:
    lo = _result(plan.lo, LO_FACTOR, device, None)
    if config.order is DISOrder.LO:
        return lo
    seed = plan.seed
    per_quark = [_sum_results([_result(j, q.charge**2, device, None) for j in jobs], seed)
                 for q, jobs in zip(config.quarks, plan.dip)]
    dip = _scale_result(_sum_results(per_quark, seed), DIP_FACTOR)
    if plan.qg_fixed:
        per_quark = [_result(j, q.charge**2, device, None) for q, j in zip(config.quarks, plan.qg_fixed)]
    else:
        per_quark = [_sum_results([_result(j, q.charge**2, device, None) for j in jobs], seed + 100)
                     for q, jobs in zip(config.quarks, plan.qg)]
    qg = _scale_result(_sum_results(per_quark, seed + 100), QG_FACTOR)
    return _sum_results((lo, dip, qg), seed)


def _sf_factor(Q2: float, config: DISConfig) -> float:
    return Q2 / (4 * math.pi**2 * AlphaEM) * config.transverse_area


# ----------------------------------------------------------------------------- public API


def photon_proton_cross_section_LO_d2b(Q2: torch.Tensor, xbj: torch.Tensor, polarization: Polarization,
                                       dipole: Dipole, config: DISConfig, *, quadrature_points: int = 24,
                                       batch_size: int = 65_536) -> IntegralResult:
    _validate_kinematics(Q2, xbj)
    engine = _Engine(dipole, config, _device(Q2))
    job = _plan_lo(engine, float(Q2), float(xbj), polarization, quadrature_points)
    engine.run()
    return _result(job, LO_FACTOR, engine.device, None)


def sigma_dip_d2b(Q2: torch.Tensor, xbj: torch.Tensor, polarization: Polarization, dipole: Dipole,
                  config: DISConfig, *, quadrature_points: int = 24, batch_size: int = 65_536,
                  seed: int = 0, **options) -> IntegralResult:
    _validate_kinematics(Q2, xbj)
    nlo = DISConfig(**{**{f: getattr(config, f) for f in config.__dataclass_fields__}, "order": DISOrder.NLO})
    engine = _Engine(dipole, nlo, _device(Q2))
    plan = _plan_sigma(engine, float(Q2), float(xbj), polarization, seed=seed, points=quadrature_points,
                       overrides=_integration_overrides(options))
    engine.jobs = [j for jobs in plan.dip for j in jobs]
    engine.run()
    per_quark = [_sum_results([_result(j, q.charge**2, engine.device, None) for j in jobs], seed)
                 for q, jobs in zip(config.quarks, plan.dip)]
    return _scale_result(_sum_results(per_quark, seed), DIP_FACTOR)


def sigma_qg_d2b(Q2: torch.Tensor, xbj: torch.Tensor, polarization: Polarization, dipole: Dipole,
                 config: DISConfig, *, batch_size: int = 65_536, seed: int = 0, **options) -> IntegralResult:
    _validate_kinematics(Q2, xbj)
    nlo = DISConfig(**{**{f: getattr(config, f) for f in config.__dataclass_fields__}, "order": DISOrder.NLO})
    engine = _Engine(dipole, nlo, _device(Q2))
    plan = _plan_sigma(engine, float(Q2), float(xbj), polarization, seed=seed - 100, points=24,
                       overrides=_integration_overrides(options), fixed=Q2.dtype == torch.float32)
    engine.jobs = list(plan.qg_fixed) + [j for jobs in plan.qg for j in jobs]
    _run_with_fallback(engine, [plan])
    if plan.qg_fixed:
        per_quark = [_result(j, q.charge**2, engine.device, None) for q, j in zip(config.quarks, plan.qg_fixed)]
    else:
        per_quark = [_sum_results([_result(j, q.charge**2, engine.device, None) for j in jobs], seed)
                     for q, jobs in zip(config.quarks, plan.qg)]
    return _scale_result(_sum_results(per_quark, seed), QG_FACTOR)


def photon_proton_cross_section_d2b(Q2: torch.Tensor, xbj: torch.Tensor, polarization: Polarization,
                                    dipole: Dipole, config: DISConfig, *, quadrature_points: int = 24,
                                    batch_size: int = 65_536, seed: int = 0, **options) -> IntegralResult:
    _validate_kinematics(Q2, xbj)
    engine = _Engine(dipole, config, _device(Q2))
    plan = _plan_sigma(engine, float(Q2), float(xbj), polarization, seed=seed, points=quadrature_points,
                       overrides=_integration_overrides(options), fixed=Q2.dtype == torch.float32)
    _run_with_fallback(engine, [plan])
    return _sigma_result(plan, config, engine.device)


def FL(Q2: torch.Tensor, xbj: torch.Tensor, dipole: Dipole, config: DISConfig, **integration_options) -> IntegralResult:
    sigma = photon_proton_cross_section_d2b(Q2, xbj, Polarization.L, dipole, config, **integration_options)
    return _scale_result(sigma, _sf_factor(float(Q2), config))


def FT(Q2: torch.Tensor, xbj: torch.Tensor, dipole: Dipole, config: DISConfig, **integration_options) -> IntegralResult:
    sigma = photon_proton_cross_section_d2b(Q2, xbj, Polarization.T, dipole, config, **integration_options)
    return _scale_result(sigma, _sf_factor(float(Q2), config))


def _two_polarisations(Q2: torch.Tensor, xbj: torch.Tensor, dipole: Dipole, config: DISConfig,
                       options: dict) -> tuple[IntegralResult, IntegralResult]:
    """F_T and F_L of one point in one engine run, with F2's seed rule (F_L gets seed + 1000
    when a seed is given, dis/observables.py:581-599)."""
    _validate_kinematics(Q2, xbj)
    options_T = dict(options)
    options_L = dict(options)
    if "seed" in options_L:
        options_L["seed"] += 1_000
    engine = _Engine(dipole, config, _device(Q2))
    plans = []
    for pol, opts in ((Polarization.T, options_T), (Polarization.L, options_L)):
        plans.append(_plan_sigma(engine, float(Q2), float(xbj), pol, seed=opts.get("seed", 0),
                                 points=opts.get("quadrature_points", 24), overrides=_integration_overrides(opts),
                                 fixed=Q2.dtype == torch.float32))
    _run_with_fallback(engine, plans)
    factor = _sf_factor(float(Q2), config)
    return tuple(_scale_result(_sigma_result(p, config, engine.device), factor) for p in plans)


def F2(Q2: torch.Tensor, xbj: torch.Tensor, dipole: Dipole, config: DISConfig, **integration_options) -> IntegralResult:
    result_T, result_L = _two_polarisations(Q2, xbj, dipole, config, integration_options)
    return _sum_results((result_T, result_L), integration_options.get("seed"))


def reduced_cross_section_y(Q2: float, xbj: float, sqrt_s: float) -> float:
    return Q2 / (sqrt_s**2 * xbj)


def sigma_r(Q2: torch.Tensor, xbj: torch.Tensor, dipole: Dipole, config: DISConfig, *, sqrt_s: float = 318.0,
            **integration_options) -> IntegralResult:
    """Reduced cross section sigma_r = F2 - y^2/(1 + (1-y)^2) F_L with y = Q^2/(s x_Bj)
    (no counterpart in the reference package, which stops at F2 and F_L)."""
    result_T, result_L = _two_polarisations(Q2, xbj, dipole, config, integration_options)
    y = reduced_cross_section_y(float(Q2), float(xbj), sqrt_s)
    f = y * y / (1 + (1 - y) ** 2)
    value = result_T.value + (1 - f) * result_L.value
    error = torch.sqrt(result_T.error.square() + ((1 - f) * result_L.error).square())
    return IntegralResult(value, error, result_T.n_eval + result_L.n_eval,
                          result_T.converged and result_L.converged, integration_options.get("seed"))


def structure_functions(Q2: torch.Tensor, xbj: torch.Tensor, dipole: Dipole, config: DISConfig, *,
                        sqrt_s: float | None = None, seed: int = 0, quadrature_points: int = 24,
                        fixed_sobol: bool | None = None, **options) -> dict[str, torch.Tensor]:
    """F_T, F_L, F_2 (and sigma_r when sqrt_s is given) for many (Q^2, x_Bj) points in one
    batched device run.  Every point uses the single-point functions' seeds (F_T: seed,
    F_L: seed + 1000), so each entry equals F2(Q2[i], xbj[i], ..., seed=seed) run alone."""
    Q2h = torch.as_tensor(Q2, dtype=torch.float64).reshape(-1).cpu()
    xh = torch.as_tensor(xbj, dtype=torch.float64).reshape(-1).cpu()
    if Q2h.numel() != xh.numel():
        raise ValueError("Q2 and xbj must have the same number of points")
    if bool((Q2h <= 0).any()) or bool(((xh <= 0) | (xh > 1)).any()):
        raise ValueError("Q2 must be positive and xbj must lie in (0, 1]")
    device = _device(Q2 if isinstance(Q2, torch.Tensor) else None)
    engine = _Engine(dipole, config, device)
    overrides = _integration_overrides(options)
    # the fixed-Sobol qqbar-g path follows the single-point rule: GBW and the mixed build
    fixed = (config.precision == "mixed") if fixed_sobol is None else fixed_sobol
    plans = []
    for i in range(Q2h.numel()):
        q2, x = float(Q2h[i]), float(xh[i])
        plans.append((_plan_sigma(engine, q2, x, Polarization.T, seed=seed, points=quadrature_points,
                                  overrides=overrides, fixed=fixed),
                      _plan_sigma(engine, q2, x, Polarization.L, seed=seed + 1000, points=quadrature_points,
                                  overrides=overrides, fixed=fixed)))
    _run_with_fallback(engine, [p for pair in plans for p in pair])
    out = {k: torch.empty(Q2h.numel(), dtype=torch.float64) for k in ("FT", "FL", "F2", "FT_error", "FL_error",
                                                                      "F2_error")}
    for i, (pt, pl) in enumerate(plans):
        factor = _sf_factor(float(Q2h[i]), config)
        rt = _scale_result(_sigma_result(pt, config, torch.device("cpu")), factor)
        rl = _scale_result(_sigma_result(pl, config, torch.device("cpu")), factor)
        out["FT"][i], out["FL"][i] = rt.value, rl.value
        out["FT_error"][i], out["FL_error"][i] = rt.error, rl.error
        out["F2"][i] = rt.value + rl.value
        out["F2_error"][i] = math.hypot(float(rt.error), float(rl.error))
    if sqrt_s is not None:
        y = Q2h / (sqrt_s**2 * xh)
        f = y * y / (1 + (1 - y) ** 2)
        out["sigma_r"] = out["FT"] + (1 - f) * out["FL"]
        out["sigma_r_error"] = torch.sqrt(out["FT_error"] ** 2 + ((1 - f) * out["FL_error"]) ** 2)
    return {k: v.to(device) for k, v in out.items()}


def structure_functions_many(Q2, xbj, dipoles, config: DISConfig, *, sqrt_s: float | None = None, seed: int = 0,
                             seeds=None, options=None, quadrature_points: int = 24,
                             fixed_sobol: bool | None = None, **common_options) -> dict[str, torch.Tensor]:
    """``structure_functions`` for points of different dipoles (``dipoles[i]`` is point i's:
    e.g. the tables of many parameter sets or requests) in one batched device run: every term
    of every point goes into the same few launches whatever its dipole.  ``seeds[i]`` and
    ``options[i]`` (dicts of the integration keywords) override ``seed`` and the common
    keywords per point; points whose integration settings agree share the launches.  Entry
    i equals ``structure_functions(Q2[i], xbj[i], dipoles[i], ..., seed=seeds[i],
    **options[i])`` run alone."""
    Q2h = [float(v) for v in torch.as_tensor(Q2, dtype=torch.float64).reshape(-1).tolist()]
    xh = [float(v) for v in torch.as_tensor(xbj, dtype=torch.float64).reshape(-1).tolist()]
    if not (len(Q2h) == len(xh) == len(dipoles)):
        raise ValueError("Q2, xbj and dipoles must have one entry per point")
    if not Q2h:
        raise ValueError("at least one point is required")
    if any(q <= 0 for q in Q2h) or any(not 0 < x <= 1 for x in xh):
        raise ValueError("Q2 must be positive and xbj must lie in (0, 1]")
    first = dipoles[0]
    device = first.device if isinstance(first, BKDipole) else _device(Q2 if isinstance(Q2, torch.Tensor) else None)
    engine = _Engine(first, config, device)
    n = len(Q2h)
    seeds = [seed] * n if seeds is None else [int(v) for v in seeds]
    per_point = [common_options] * n if options is None else [dict(common_options, **o) for o in options]
    if len(seeds) != n or len(per_point) != n:
        raise ValueError("seeds and options need one entry per point")
    fixed = (config.precision == "mixed") if fixed_sobol is None else fixed_sobol
    plans = []
    for q2, x, d, sd, opts in zip(Q2h, xh, dipoles, seeds, per_point):
        overrides = _integration_overrides(opts)
        plans.append((_plan_sigma(engine, q2, x, Polarization.T, seed=sd, points=quadrature_points,
                                  overrides=overrides, fixed=fixed, dipole=d),
                      _plan_sigma(engine, q2, x, Polarization.L, seed=sd + 1000, points=quadrature_points,
                                  overrides=overrides, fixed=fixed, dipole=d)))
    _run_with_fallback(engine, [p for pair in plans for p in pair])
    out = {k: torch.empty(n, dtype=torch.float64) for k in ("FT", "FL", "F2", "FT_error", "FL_error", "F2_error")}
    for i, (pt, pl) in enumerate(plans):
        factor = _sf_factor(Q2h[i], config)
        rt = _scale_result(_sigma_result(pt, config, torch.device("cpu")), factor)
        rl = _scale_result(_sigma_result(pl, config, torch.device("cpu")), factor)
        out["FT"][i], out["FL"][i] = rt.value, rl.value
        out["FT_error"][i], out["FL_error"][i] = rt.error, rl.error
        out["F2"][i] = rt.value + rl.value
        out["F2_error"][i] = math.hypot(float(rt.error), float(rl.error))
    if sqrt_s is not None:
        q2t, xt = torch.tensor(Q2h, dtype=torch.float64), torch.tensor(xh, dtype=torch.float64)
        y = q2t / (sqrt_s**2 * xt)
        f = y * y / (1 + (1 - y) ** 2)
        out["sigma_r"] = out["FT"] + (1 - f) * out["FL"]
        out["sigma_r_error"] = torch.sqrt(out["FT_error"] ** 2 + ((1 - f) * out["FL_error"]) ** 2)
    return {k: v.to(device) for k, v in out.items()}


def structure_function_batch(points, dipole: Dipole, config: DISConfig, *, quadrature_points: int = 24,
                             single_precision: bool = False, **options) -> list[IntegralResult]:
    """F_T or F_L of many points in one batched device run.

    ``points`` holds (Q^2, x_Bj, polarization, seed) tuples; entry i equals
    ``FT(Q2, xbj, dipole, config, seed=seed)`` (``FL`` for Polarization.L) run alone, with
    ``single_precision`` standing for float32 Q^2 (the fixed-Sobol qqbar-g path of
    dis/observables.py:644-660).  All points share one engine, so every term of every point
    is integrated by the same few batched launches."""
    points = [(float(q2), float(x), pol, int(seed)) for q2, x, pol, seed in points]
    for q2, x, _, _ in points:
        if not q2 > 0 or not 0 < x <= 1:
            raise ValueError("Q2 must be positive and xbj must lie in (0, 1]")
    device = dipole.device if isinstance(dipole, BKDipole) else _device()
    engine = _Engine(dipole, config, device)
    overrides = _integration_overrides(options)
    plans = [_plan_sigma(engine, q2, x, pol, seed=seed, points=quadrature_points, overrides=overrides,
                         fixed=single_precision) for q2, x, pol, seed in points]
    _run_with_fallback(engine, plans)
    return [_scale_result(_sigma_result(plan, config, device), _sf_factor(q2, config))
            for plan, (q2, _, _, _) in zip(plans, points)]


# ----------------------------------------------------------------------------- integrands


def _integrand(term: int, x: torch.Tensor, kin: _native.DisKinematics, dipole: Dipole, config: DISConfig,
               precision: int | None = None) -> torch.Tensor:
    _native.require_cuda(x, "x")
    dims = _native.DIS_DIMS[term]
    if x.ndim != 2 or x.shape[1] != dims:
        raise ValueError(f"the term takes points of {dims} dimensions")
    x64 = x.to(torch.float64).contiguous()
    out = torch.empty(x64.shape[0], dtype=torch.float64, device=x.device)
    if precision is None:
        precision = _native.PRECISION_FP64 if x.dtype == torch.float64 else _native.PRECISION_MIXED
    lib = _native.load()
    import ctypes

    with torch.cuda.device(x.device):
        _native.check(lib.nlo_dis_integrand(ctypes.byref(kin), term, ctypes.byref(dipole.native()),
                                            config.cuda_nested_points, precision, x64.data_ptr(), x64.shape[0],
                                            out.data_ptr(), _native.stream_handle(x.device)))
    return out.to(x.dtype)


def integrand_dip_massive(x: torch.Tensor, Q2: torch.Tensor, xbj: torch.Tensor, polarization: Polarization,
                          quark: Quark, contribution: str, dipole: Dipole, config: DISConfig) -> torch.Tensor:
    order = _DIP_CONTRIBUTIONS[polarization].index(contribution) if contribution in _DIP_CONTRIBUTIONS[
        polarization] else None
    if order is None or x.shape[1] != 2 + order:
        raise ValueError(f"invalid contribution/dimension pair: {polarization}, {contribution}, {x.shape[1]}")
    kin = kinematics(float(Q2), float(xbj), polarization, config, quark)
    return _integrand(TERMS[f"DIP{order}"], x, kin, dipole, config)


def integrand_qgunsub_massive(x: torch.Tensor, Q2: torch.Tensor, xbj: torch.Tensor, polarization: Polarization,
                              quark: Quark, contribution: str, dipole: Dipole, config: DISConfig) -> torch.Tensor:
    dims = {"I1": 5, "I2": 6, "I3": 7}.get(contribution)
    if dims is None or x.shape[1] != dims:
        raise ValueError(f"invalid qqg contribution/dimension pair: {contribution}, {x.shape[1]}")
    kin = kinematics(float(Q2), float(xbj), polarization, config, quark)
    return _integrand(TERMS[contribution], x, kin, dipole, config)


def integrand_qg_nested_massive(x: torch.Tensor, Q2: torch.Tensor, xbj: torch.Tensor, polarization: Polarization,
                                quark: Quark, contribution: str, dipole: Dipole, config: DISConfig) -> torch.Tensor:
    if contribution not in {"I2", "I3"} or x.shape[1] != 5:
        raise ValueError(f"invalid nested qqg contribution/dimension pair: {contribution}, {x.shape[1]}")
    kin = kinematics(float(Q2), float(xbj), polarization, config, quark)
    return _integrand(TERMS[contribution + "N"], x, kin, dipole, config)


__all__ = [
    "F2",
    "FL",
    "FT",
    "integrand_dip_massive",
    "integrand_qg_nested_massive",
    "integrand_qgunsub_massive",
    "kinematics",
    "photon_proton_cross_section_LO_d2b",
    "photon_proton_cross_section_d2b",
    "sigma_dip_d2b",
    "sigma_qg_d2b",
    "sigma_r",
    "structure_functions",
]
