"""CPU FP64 oracle for the NLO BK hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker: ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import it to compute reference values on the
same inputs the CUDA product consumes.  The product package
``nlo_bk_optimized_b200`` never imports it.

The numerics live in ``nlo_oracle.c`` (a plain-C restatement of the reference
``torch_nlo_clean/src/nlo_torch`` BK path; see its header for the file:line map).
This module wraps it with ctypes and adds the Python-level orchestration of
the reference's evolution driver:

* ``derivative``   -- dN/dY assembly, bk/evolution.py:329-351 and 354-488
                      (K1 by the fixed rule of custom_kernels/bk/k1/kernel.cu:2040-2092,
                      K2+Kf by quasi-Monte Carlo on fixed Sobol points)
* ``derivative_shard`` -- one shard's part of it (K1 by parent, K2+Kf by point range),
                      for the multi-rank evolution (no counterpart in the reference)
* ``vegas_k2kf`` / ``derivative_vegas`` -- K2+Kf by Vegas per parent with grid reuse
                      (bk/derivatives.py:389-421, numerics/integration.py:120-589,
                      bk/evolution.py:354-424)
* ``evolve``       -- stepping loop bk/evolution.py:85-159 with the Euler
                      (:110-122), Kutta RK3 (:190-236) or classical RK4 stepper
* ``r_grid``       -- bk/evolution.py:584-592
* ``mv_amplitude`` -- bk/initial_conditions.py:29-35
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from oracle import build as _build

_lib = None


class Physics(ctypes.Structure):
    _fields_ = [
        ("nc", ctypes.c_double),
        ("nf", ctypes.c_double),
        ("lambda_qcd", ctypes.c_double),
        ("c2", ctypes.c_double),
        ("minr", ctypes.c_double),
        ("ksub", ctypes.c_double),
        ("symmetrize", ctypes.c_int),
        ("fixed_coupling", ctypes.c_int),
        ("fixed_alpha_s", ctypes.c_double),
        ("alpha_cap", ctypes.c_double),
        ("order", ctypes.c_int),
        ("rc_lo", ctypes.c_int),
        ("resum_rc", ctypes.c_int),
        ("rc_nlo", ctypes.c_int),
    ]


# enum codes of or_physics (nlo_oracle.c), by the reference's enum member names
ORDER = {"NLO_RESUM_DLOG_SLOG": 0, "NLO_RESUM_DLOG": 1, "NLO": 2, "LO_RESUM_DLOG_SLOG": 3, "LO_RESUM_DLOG": 4,
         "LO": 5}
RC_LO = {"BALITSKY_LO": 0, "FIXED_LO": 0, "PARENT_LO": 1, "SMALLEST_LO": 2, "FAC_LO": 3, "BEUF_LO": 4}
RESUM_RC = {"RESUM_RC_SMALLEST": 0, "RESUM_RC_PARENT": 1, "RESUM_RC_FIXED": 2}
RC_NLO = {"SMALLEST_NLO": 0, "FIXED_NLO": 0, "PARENT_NLO": 1}


class _Spline(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int),
        ("x", ctypes.POINTER(ctypes.c_double)),
        ("a", ctypes.POINTER(ctypes.c_double)),
        ("b", ctypes.POINTER(ctypes.c_double)),
        ("c", ctypes.POINTER(ctypes.c_double)),
        ("d", ctypes.POINTER(ctypes.c_double)),
        ("rmin", ctypes.c_double),
        ("rmax", ctypes.c_double),
    ]


def _dp(array: np.ndarray):
    return array.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = _build.build()
        handle = ctypes.CDLL(str(path))
        D, I, P = ctypes.c_double, ctypes.c_int, ctypes.POINTER
        DP = P(D)
        handle.or_alpha_s.restype = D
        handle.or_alpha_s.argtypes = [D, P(Physics)]
        handle.or_natural_spline.argtypes = [DP, DP, I, DP, DP, DP, DP]
        handle.or_loglog_knots.argtypes = [DP, I, I, I, DP]
        handle.or_n_from_nspline.restype = D
        handle.or_n_from_nspline.argtypes = [P(_Spline), D]
        handle.or_n_from_sspline.restype = D
        handle.or_n_from_sspline.argtypes = [P(_Spline), D]
        handle.or_k1_integrand.restype = D
        handle.or_k1_integrand.argtypes = [D, D, D, P(_Spline), P(Physics)]
        handle.or_bessel_i1.restype = D
        handle.or_bessel_i1.argtypes = [D]
        handle.or_k1_fixed_many.argtypes = [DP, I, P(_Spline), P(Physics), DP, DP, DP, DP, DP]
        handle.or_k1_fixed_history_many.argtypes = [DP, I, P(_Spline), P(Physics), DP, DP, DP, DP, DP, I, DP, DP, I,
                                                    DP]
        handle.or_k1_integrand_history.restype = D
        handle.or_k1_integrand_history.argtypes = [D, D, D, P(_Spline), P(Physics), DP, I, DP, DP, I]
        handle.or_nlo_kernels.argtypes = [D, D, D, D, D, D, D, DP]
        handle.or_k2kf_integrand.argtypes = [D, DP, P(_Spline), P(Physics), DP]
        handle.or_k2kf_sums.argtypes = [DP, I, DP, ctypes.c_long, DP, DP, I, P(_Spline), P(Physics), DP]
        handle.or_k2kf_values.argtypes = [D, DP, ctypes.c_long, P(_Spline), P(Physics), DP, DP]
        handle.or_sobol.argtypes = [
            P(ctypes.c_int64), P(ctypes.c_int64), I, ctypes.c_long, ctypes.c_long, I, DP
        ]
        handle.or_nlo_kernels_literal_q.argtypes = [D, D, D, D, D, D, D, DP]
        handle.or_lo_kernel_literal_q.restype = D
        handle.or_lo_kernel_literal_q.argtypes = [D, D, D, P(Physics)]
        handle.or_lo_kernel.restype = D
        handle.or_lo_kernel.argtypes = [D, D, D, P(Physics)]
        handle.or_k1_dipole.restype = D
        handle.or_k1_dipole.argtypes = [P(_Spline), D, D, D]
        handle.or_k1_dipole_literal_q.restype = D
        handle.or_k1_dipole_literal_q.argtypes = [P(_Spline), D, D, D]
        handle.or_k2_dipoles.argtypes = [P(_Spline), D, DP, DP, DP]
        handle.or_num_threads.restype = I
        _lib = handle
    return _lib


def physics(config) -> Physics:
    """Physics constants and switches from any object with BKConfig's field names
    (enum members are read by name, so the reference's own BKConfig works too)."""

    def name(field, default):
        value = getattr(config, field, None)
        return getattr(value, "name", default)

    fixed_coupling = name("RC_LO", "") == "FIXED_LO" or name("RC_NLO", "") == "FIXED_NLO"
    return Physics(
        float(config.NC),
        float(config.NF),
        float(config.LambdaQCD),
        float(config.C2),
        float(config.MINR),
        float(config.KSUB),
        int(bool(config.SYMMETRIZE_Z_Z2_INTEGRATION)),
        int(fixed_coupling),
        float(config.FIXED_AS),
        float(getattr(config, "ALPHA_S_CAP", 0.0) or 0.0),
        ORDER[name("Order", "NLO_RESUM_DLOG_SLOG")],
        RC_LO[name("RC_LO", "BALITSKY_LO")],
        RESUM_RC[name("RESUM_RC", "RESUM_RC_SMALLEST")],
        RC_NLO[name("RC_NLO", "SMALLEST_NLO")],
    )


def has_nlo_kernels(phys: Physics) -> bool:
    """Order.has_nlo_kernels (bk/config.py:44-50)."""
    return phys.order <= ORDER["NLO"]


@dataclass
class Spline:
    """Natural cubic spline of a log-log table over the r grid."""

    x: np.ndarray
    a: np.ndarray
    b: np.ndarray
    c: np.ndarray
    d: np.ndarray
    rmin: float
    rmax: float

    def struct(self) -> _Spline:
        s = _Spline()
        s.n = self.x.size
        s.x, s.a, s.b, s.c, s.d = (_dp(v) for v in (self.x, self.a, self.b, self.c, self.d))
        s.rmin, s.rmax = self.rmin, self.rmax
        self._keep = s
        return s


def r_grid(minr: float, maxr: float, rpoints: int) -> np.ndarray:
    """bk/evolution.py:584-592, float64 (torch.pow per index, as the reference)."""

    import torch

    rind = torch.arange(rpoints + 1, dtype=torch.float64)
    step = (maxr / minr) ** (1 / rpoints)
    return (minr * torch.pow(rind.new_tensor(step), rind)).numpy().copy()


def mv_amplitude(r: np.ndarray, qs0sqr: float, ec: float = 1.0, lambdaqcd: float = 0.241,
                 gamma: float = 1.0) -> np.ndarray:
    """bk/initial_conditions.py:29-35."""

    exponent = np.power(r * r * qs0sqr, gamma) / 4 * np.log(1 / (r * lambdaqcd) + ec * 2.7182818)
    return np.where(exponent < 1e-5, exponent, 1 - np.exp(-exponent))


def loglog_spline(r: np.ndarray, N: np.ndarray, kind: int, force_positive: bool = True) -> Spline:
    """kind 0: log N spline (K1); kind 1: log S spline (K2+Kf)."""

    r = np.ascontiguousarray(r, dtype=np.float64)
    N = np.ascontiguousarray(N, dtype=np.float64)
    n = r.size
    x = np.log(r)
    y = np.empty(n)
    lib().or_loglog_knots(_dp(N), n, kind, int(force_positive), _dp(y))
    a, b, c, d = (np.empty(n - 1) for _ in range(4))
    lib().or_natural_spline(_dp(x), _dp(y), n, _dp(a), _dp(b), _dp(c), _dp(d))
    return Spline(x, a, b, c, d, float(r[0]), float(r[-1]))


def natural_spline(x: np.ndarray, y: np.ndarray):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = x.size
    a, b, c, d = (np.empty(n - 1) for _ in range(4))
    lib().or_natural_spline(_dp(x), _dp(y), n, _dp(a), _dp(b), _dp(c), _dp(d))
    return a, b, c, d


def gauss_legendre(order: int) -> tuple[np.ndarray, np.ndarray]:
    x, w = np.polynomial.legendre.leggauss(order)
    return np.ascontiguousarray(x), np.ascontiguousarray(w)


def _history_arrays(r: np.ndarray, history) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    hy = np.ascontiguousarray(history[0], dtype=np.float64)
    hN = np.ascontiguousarray(history[1], dtype=np.float64)
    rg = np.ascontiguousarray(r, dtype=np.float64)
    if hN.ndim != 2 or hN.shape != (hy.size, rg.size):
        raise ValueError("history must be (y [rows], N [rows, R])")
    return rg, hy, hN


def k1_fixed(rpar: np.ndarray, nspline: Spline, phys: Physics, history=None, r_grid=None) -> np.ndarray:
    """The fixed K1 rule at the parents rpar; with ``history`` = (y [rows], N [rows, R]) on
    ``r_grid``, the kinematical constraint's K1 (the last row the current amplitude)."""
    rpar = np.ascontiguousarray(rpar, dtype=np.float64)
    x8, w8 = gauss_legendre(8)
    x24, w24 = gauss_legendre(24)
    out = np.empty(rpar.size)
    if history is None:
        lib().or_k1_fixed_many(_dp(rpar), rpar.size, ctypes.byref(nspline.struct()), ctypes.byref(phys),
                               _dp(x8), _dp(w8), _dp(x24), _dp(w24), _dp(out))
        return out
    rg, hy, hN = _history_arrays(r_grid, history)
    lib().or_k1_fixed_history_many(_dp(rpar), rpar.size, ctypes.byref(nspline.struct()), ctypes.byref(phys),
                                   _dp(x8), _dp(w8), _dp(x24), _dp(w24), _dp(rg), rg.size, _dp(hy), _dp(hN),
                                   hy.size, _dp(out))
    return out


def k1_integrand(r: float, z: float, theta: float, nspline: Spline, phys: Physics, history=None,
                 r_grid=None) -> float:
    if history is None:
        return lib().or_k1_integrand(r, z, theta, ctypes.byref(nspline.struct()), ctypes.byref(phys))
    rg, hy, hN = _history_arrays(r_grid, history)
    return lib().or_k1_integrand_history(r, z, theta, ctypes.byref(nspline.struct()), ctypes.byref(phys), _dp(rg),
                                         rg.size, _dp(hy), _dp(hN), hy.size)


def k2kf_integrand(r: float, x: np.ndarray, sspline: Spline, phys: Physics) -> tuple[float, float]:
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(2)
    lib().or_k2kf_integrand(r, _dp(x), ctypes.byref(sspline.struct()), ctypes.byref(phys), _dp(out))
    return float(out[0]), float(out[1])


def k2kf_sums(rpar: np.ndarray, points: np.ndarray, lower: np.ndarray, width: np.ndarray, map_f32: bool,
              sspline: Spline, phys: Physics) -> np.ndarray:
    """Per-parent [sum K2 w, sum Kf w, sum (K2+Kf)^2 w^2] over unit-cube points [n,4]."""

    rpar = np.ascontiguousarray(rpar, dtype=np.float64)
    points = np.ascontiguousarray(points, dtype=np.float64)
    lower = np.ascontiguousarray(lower, dtype=np.float64)
    width = np.ascontiguousarray(width, dtype=np.float64)
    out = np.empty((rpar.size, 3))
    lib().or_k2kf_sums(_dp(rpar), rpar.size, _dp(points), points.shape[0], _dp(lower), _dp(width),
                       int(map_f32), ctypes.byref(sspline.struct()), ctypes.byref(phys), _dp(out))
    return out


def sobol(state: np.ndarray, shift: np.ndarray, offset: int, n: int, as_f32: bool) -> np.ndarray:
    state = np.ascontiguousarray(state, dtype=np.int64)
    shift = np.ascontiguousarray(shift, dtype=np.int64)
    dims = shift.size
    out = np.empty((n, dims))
    lib().or_sobol(state.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                   shift.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), dims, offset, n, int(as_f32),
                   _dp(out))
    return out


def sobol_state(dims: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Scrambled direction numbers and shift of SobolEngine(dims, scramble=True, seed)."""

    import torch

    engine = torch.quasirandom.SobolEngine(dims, scramble=True, seed=seed)
    return engine.sobolstate.numpy().copy(), engine.shift.numpy().copy()


def nlo_kernels(r, lz, lz2, th, th2, nf=3.0, nc=3.0) -> np.ndarray:
    out = np.empty(3)
    lib().or_nlo_kernels(r, lz, lz2, th, th2, nf, nc, _dp(out))
    return out


def nlo_kernels_literal_quad(r, lz, lz2, th, th2, nf=3.0, nc=3.0) -> np.ndarray:
    out = np.empty(3)
    lib().or_nlo_kernels_literal_q(r, lz, lz2, th, th2, nf, nc, _dp(out))
    return out


def lo_kernel(r, z, theta, phys: Physics) -> float:
    return lib().or_lo_kernel(r, z, theta, ctypes.byref(phys))


def lo_kernel_literal_quad(r, z, theta, phys: Physics) -> float:
    return lib().or_lo_kernel_literal_q(r, z, theta, ctypes.byref(phys))


def k1_dipole(nspline: Spline, r: float, z: float, theta: float) -> tuple[float, float]:
    """(stable FP64, quad literal) K1 dipole factor."""

    st = nspline.struct()
    return (lib().or_k1_dipole(ctypes.byref(st), r, z, theta),
            lib().or_k1_dipole_literal_q(ctypes.byref(st), r, z, theta))


def k2_dipoles(sspline: Spline, r: float, x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(stable FP64, quad literal) [dipole, dipole_swap, fermion factor] of the K2+Kf integrand."""

    x = np.ascontiguousarray(x, dtype=np.float64)
    out, out_q = np.empty(3), np.empty(3)
    lib().or_k2_dipoles(ctypes.byref(sspline.struct()), r, _dp(x), _dp(out), _dp(out_q))
    return out, out_q


def bessel_i1(x: float) -> float:
    return lib().or_bessel_i1(x)


def alpha_s(r: float, phys: Physics) -> float:
    return lib().or_alpha_s(r, ctypes.byref(phys))


def num_threads() -> int:
    return lib().or_num_threads()


def nlo_box(r: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """bk/derivatives.py:424-431: [log(r0/2), log(2 r_max)]^2 x [0, 2 pi]^2 as (lower, width)."""

    lo = math.log(0.5 * r[0])
    hi = math.log(2 * r[-1])
    lower = np.array([lo, lo, 0.0, 0.0])
    width = np.array([hi - lo, hi - lo, 2 * math.pi, 2 * math.pi])
    return lower, width


@dataclass
class Derivative:
    dNdy: np.ndarray
    K1: np.ndarray
    K2: np.ndarray
    Kf: np.ndarray
    sq: np.ndarray


def derivative(N: np.ndarray, r: np.ndarray, phys: Physics, points: np.ndarray, map_f32: bool,
               force_positive: bool = True, history=None) -> Derivative:
    """dN/dY = K1 + (K2+Kf) at active parents (index > 0 and N <= 0.99999), else 0;
    non-finite values become 0 (bk/evolution.py:329-351, 501).  ``history`` = (y, N rows)
    gives K1 the kinematical constraint (its last row is N)."""

    nspl = loglog_spline(r, N, 0, force_positive)
    sspl = loglog_spline(r, N, 1, force_positive)
    active = np.nonzero((np.arange(r.size) > 0) & (N <= 0.99999))[0]
    K1 = np.zeros_like(N)
    K2 = np.zeros_like(N)
    Kf = np.zeros_like(N)
    sq = np.zeros_like(N)
    if active.size:
        K1[active] = k1_fixed(r[active], nspl, phys, history=history, r_grid=r)
        if has_nlo_kernels(phys):  # LO orders take no K2 + Kf (bk/evolution.py:391, 473)
            lower, width = nlo_box(r)
            sums = k2kf_sums(r[active], points, lower, width, map_f32, sspl, phys)
            n = points.shape[0]
            K2[active] = sums[:, 0] / n
            Kf[active] = sums[:, 1] / n
            sq[active] = sums[:, 2]
    dNdy = K1 + K2 + Kf
    dNdy = np.where(np.isfinite(dNdy), dNdy, 0.0)
    return Derivative(dNdy, K1, K2, Kf, sq)


def derivative_shard(N: np.ndarray, r: np.ndarray, phys: Physics, points: np.ndarray, map_f32: bool, shard: int,
                     shards: int, force_positive: bool = True) -> np.ndarray:
    """One shard's part of ``derivative``: K1 of the active parents i with i % shards == shard,
    plus K2+Kf of every active parent summed over the shard's points
    [shard n / shards, (shard + 1) n / shards) and divided by the total n; the shards' parts
    add up to ``derivative(...).dNdy``."""

    nspl = loglog_spline(r, N, 0, force_positive)
    sspl = loglog_spline(r, N, 1, force_positive)
    active = np.nonzero((np.arange(r.size) > 0) & (N <= 0.99999))[0]
    out = np.zeros_like(N)
    if active.size:
        mine = active[active % shards == shard]
        if mine.size:
            out[mine] += k1_fixed(r[mine], nspl, phys)
        if has_nlo_kernels(phys):
            n = points.shape[0]
            lo, hi = n * shard // shards, n * (shard + 1) // shards
            if hi > lo:
                lower, width = nlo_box(r)
                sums = k2kf_sums(r[active], points[lo:hi], lower, width, map_f32, sspl, phys)
                out[active] += (sums[:, 0] + sums[:, 1]) / n
    return np.where(np.isfinite(out), out, 0.0)


def k2kf_values(r: float, x: np.ndarray, sspline: Spline, phys: Physics) -> tuple[np.ndarray, np.ndarray]:
    """_nlo_integrand x Jacobian (K2 part, Kf part) at box points x [n, 4]."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[0]
    k2, kf = np.empty(n), np.empty(n)
    lib().or_k2kf_values(r, _dp(x), n, ctypes.byref(sspline.struct()), ctypes.byref(phys), _dp(k2), _dp(kf))
    return k2, kf


@dataclass
class VegasGrid:
    """One parent's Vegas state between right-hand sides (the reference's VegasState)."""

    edges: np.ndarray | None = None
    last_components: np.ndarray | None = None
    last_error: float | None = None


@dataclass
class VegasResult:
    value: float
    error: float
    n_eval: int
    iterations: int
    converged: bool
    components: np.ndarray  # combined K2, Kf estimates
    edges: np.ndarray


def vegas_k2kf(r: float, sspline: Spline, phys: Physics, box: tuple[np.ndarray, np.ndarray], seed: int, *,
               samples: int, warmup: int, max_iterations: int = 4, min_iterations: int = 2, bins: int = 32,
               epsrel: float = 0.2, epsabs: float = 0.0, state: VegasGrid | None = None,
               reuse_warmup_fraction: float = 0.0, f32_points: bool = False) -> VegasResult:
    """vegas() of numerics/integration.py:120-589 for the K2+Kf integrand of one parent
    (rapidity_derivative_nlo, bk/derivatives.py:389-421) on the Sobol points of `seed`,
    indices 0, 1, ... across the rounds: coordinate u gives the bin floor(u bins) and the
    fraction u bins - bin.  A `state` holding edges starts from them with the warm-up
    max(2, warmup x reuse_warmup_fraction) (none when either is 0); the final edges and the
    combined K2/Kf components are written back.  f32_points rounds the box points to float32
    before the integrand (the positions the mixed device build evaluates at)."""
    from oracle import dis as odis

    lower, width = box
    volume = float(np.prod(width))
    reused = state is not None and state.edges is not None
    edges = state.edges.copy() if reused else np.tile(np.linspace(0, 1, bins + 1), (4, 1))
    if reused:
        warm = max(2, int(warmup * reuse_warmup_fraction)) if warmup > 0 and reuse_warmup_fraction > 0 else 0
    else:
        warm = warmup
    sobol_state_, sobol_shift = sobol_state(4, seed)
    offset = 0
    estimates, variances, comps = [], [], []
    n_eval, value, error, converged = 0, 0.0, 0.0, False
    rounds = max_iterations + int(warm > 0)
    for k in range(rounds):
        is_warm = warm > 0 and k == 0
        n = warm if is_warm else samples
        u = sobol(sobol_state_, sobol_shift, offset, n, as_f32=False)
        offset += n
        scaled = u * bins
        bi = np.minimum(np.floor(scaled).astype(np.int64), bins - 1)
        fr = scaled - bi
        unit, inv = odis.vegas_map(edges, bi, fr)
        x = lower + width * unit
        if f32_points:
            x = x.astype(np.float32).astype(np.float64)
        k2, kf = k2kf_values(r, x, sspline, phys)
        w_k2, w_kf = k2 * volume * inv, kf * volume * inv
        w = (k2 + kf) * volume * inv
        hist = np.zeros((4, bins))
        count = np.zeros((4, bins))
        for d in range(4):
            hist[d] = np.bincount(bi[:, d], weights=np.abs(w), minlength=bins)
            count[d] = np.bincount(bi[:, d], minlength=bins)
        n_eval += n
        edges = odis.adapt_edges(edges, hist, count)
        if is_warm:
            continue
        total, total2 = float(np.sum(w)), float(np.sum(w * w))
        est = total / n
        var = max(max(total2 - total * total / n, 0.0) / (n - 1) / n, np.finfo(np.float64).tiny)
        estimates.append(est)
        variances.append(var)
        comps.append(np.array([np.sum(w_k2) / n, np.sum(w_kf) / n]))
        wts = 1 / np.array(variances)
        value = float(np.sum(wts * np.array(estimates)) / wts.sum())
        error = float(math.sqrt(1 / wts.sum()))
        converged = len(estimates) >= min_iterations and error <= max(epsabs, epsrel * abs(value))
        if converged:
            break
    wts = 1 / np.array(variances)
    components = (wts[:, None] * np.stack(comps)).sum(axis=0) / wts.sum()
    if state is not None:
        state.edges = edges.copy()
        state.last_components = components
        state.last_error = error
    return VegasResult(value, error, n_eval, len(estimates), converged, components, edges)


def derivative_vegas(N: np.ndarray, r: np.ndarray, phys: Physics, seed: int, *, samples: int,
                     grids: dict[int, VegasGrid] | None = None, reuse_warmup_fraction: float = 0.25,
                     f32_points: bool = False, force_positive: bool = True, replicas: int = 0,
                     **options) -> dict:
    """dN/dY with K2+Kf by Vegas per active parent (_derivative_components with
    IntegrationMethod.VEGAS, bk/evolution.py:354-424): `grids` keyed by grid index are the
    per-parent states carried between calls (None: fresh grids, as without vegas_states).

    replicas > 0 (with `grids`): the replica refinement of bk/evolution.py:411-456 -- a parent
    whose condition (|K1| + |K2| + |Kf|) / max(|K1 + K2 + Kf|, 0.05 (|K1| + |K2| + |Kf|)), with
    the combined K2 and Kf estimates of its integral, is at least 4, or whose N exceeds 0.9,
    gets `replicas` more integrals on fresh grids with the seeds seed + 1000 k; its K2+Kf is
    the mean of all of them (added in the order main, replica 1, 2, ...), its components the
    mean, its error sqrt(sum error^2) / (replicas + 1); its grid stays the main integral's."""
    nspl = loglog_spline(r, N, 0, force_positive)
    sspl = loglog_spline(r, N, 1, force_positive)
    active = np.nonzero((np.arange(r.size) > 0) & (N <= 0.99999))[0]
    K1 = np.zeros_like(N)
    K2Kf = np.zeros_like(N)
    results = {}
    if active.size:
        K1[active] = k1_fixed(r[active], nspl, phys)
        if has_nlo_kernels(phys):
            box = nlo_box(r)
            for i in active:
                state = None if grids is None else grids.setdefault(int(i), VegasGrid())
                res = vegas_k2kf(float(r[i]), sspl, phys, box, seed, samples=samples,
                                 warmup=max(2, samples // 5), state=state,
                                 reuse_warmup_fraction=reuse_warmup_fraction if grids is not None else 0.0,
                                 f32_points=f32_points, **options)
                K2Kf[i] = res.value
                results[int(i)] = res
            if replicas > 0 and grids is not None:
                warm = max(2, samples // 5)
                for i in active:
                    comp = grids[int(i)].last_components
                    if comp is None:
                        continue
                    scale = abs(K1[i]) + abs(comp[0]) + abs(comp[1])
                    net = K1[i] + comp[0] + comp[1]
                    condition = scale / max(abs(net), 0.05 * scale)
                    if not (condition >= 4.0 or N[i] > 0.9):
                        continue
                    total, err2 = K2Kf[i], grids[int(i)].last_error ** 2
                    comps = [comp]
                    for k in range(1, replicas + 1):
                        rep = VegasGrid()
                        res = vegas_k2kf(float(r[i]), sspl, phys, box, seed + 1000 * k, samples=samples, warmup=warm,
                                         state=rep, f32_points=f32_points, **options)
                        total += res.value
                        err2 += res.error ** 2
                        comps.append(rep.last_components)
                    K2Kf[i] = total / (replicas + 1)
                    grids[int(i)].last_components = np.mean(np.stack(comps), axis=0)
                    grids[int(i)].last_error = math.sqrt(err2) / (replicas + 1)
    dNdy = K1 + K2Kf
    return {"dNdy": np.where(np.isfinite(dNdy), dNdy, 0.0), "K1": K1, "K2Kf": K2Kf, "vegas": results}


def evolve(N0: np.ndarray, r: np.ndarray, phys: Physics, points: np.ndarray, map_f32: bool, step: float,
           maxy: float, stepper: str = "rk4", force_positive: bool = True, kinematical_constraint: bool = False,
           abserr: float = 1e-6, relerr: float = 1e-4, eps: float = float(np.finfo(np.float64).eps)):
    """Rapidity stepping (bk/evolution.py:85-159); returns (y[steps+1], N[steps+1, R]).
    With the kinematical constraint (Euler only) each step's K1 reads the rows so far.

    stepper "rk2_adaptive": _adaptive_rk2_to (bk/evolution.py:239-326) inside every output
    step -- a midpoint step of size h against two of size h/2, error |two halves - one|/3
    against abserr + relerr |two halves|; accepted when the largest ratio is at most 1 (h then
    grows by min(5, 0.9 ratio^(-1/3)), by 5 for a zero error), else retried with h shrunk by
    max(0.1, 0.9 ratio^(-1/3)); h carries over from one output step to the next, and the
    row's rapidity is the sum of the accepted steps."""

    ys = [0.0]
    Ns = [np.array(N0, dtype=np.float64)]
    N = Ns[0].copy()
    y = 0.0
    h_adaptive = step
    if kinematical_constraint and stepper != "euler":
        raise ValueError("the kinematical constraint requires the Euler stepper")

    def f(state):
        history = (np.array(ys), np.stack(Ns)) if kinematical_constraint else None
        return derivative(state, r, phys, points, map_f32, force_positive, history=history).dNdy

    while True:
        h = step
        if stepper == "euler":
            N = N + h * f(N)
        elif stepper == "rk3":
            k1 = f(N)
            k2 = f(N + 0.5 * h * k1)
            k3 = f(N + h * (-k1 + 2.0 * k2))
            N = N + h * (k1 + 4.0 * k2 + k3) / 6.0
        elif stepper == "rk4":
            k1 = f(N)
            k2 = f(N + 0.5 * h * k1)
            k3 = f(N + 0.5 * h * k2)
            k4 = f(N + h * k3)
            N = N + h * (k1 + 2.0 * k2 + 2.0 * k3 + k4) / 6.0
        elif stepper == "rk2_adaptive":
            nexty = y + step
            while y < nexty:
                st = min(h_adaptive, nexty - y)
                k1 = f(N)
                full = N + st * f(N + 0.5 * st * k1)
                hs = st / 2
                half = N + hs * f(N + 0.5 * hs * k1)
                k1h = f(half)
                two = half + hs * f(half + 0.5 * hs * k1h)
                error = np.abs(two - full) / 3
                ratio = float(np.max(error / (abserr + relerr * np.abs(two))))
                if ratio <= 1:
                    N = two
                    y += st
                    h_adaptive = st * (5.0 if ratio == 0 else min(5.0, 0.9 * ratio ** (-1 / 3)))
                else:
                    h_adaptive = st * max(0.1, 0.9 * ratio ** (-1 / 3))
                    if h_adaptive <= eps * max(1.0, abs(y)):
                        raise RuntimeError(f"BK RK2 step underflow at y={y}")
        else:
            raise ValueError(stepper)
        if stepper != "rk2_adaptive":
            y = y + step
        if force_positive:
            N = np.clip(N, 0.0, 1.0)
        if not np.all(np.isfinite(N)):
            raise FloatingPointError(f"non-finite BK amplitude after rapidity step y={y}")
        ys.append(y)
        Ns.append(N.copy())
        if y >= maxy - 1e-12 * max(1.0, abs(maxy), abs(step)):
            break
    return np.array(ys), np.stack(Ns)
