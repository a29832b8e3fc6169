"""Operation census of the K2+Kf integrand -- test and measurement infrastructure.

The roofline of the K2+Kf kernel needs the arithmetic an evaluation costs, counted on
the algorithm rather than on any one build's instructions, so that the numerator stays
fixed while the kernel changes.  This module restates the oracle's FP64 K2+Kf path
(``k2_prepare`` and ``k2_eval`` of nlo_oracle.c, which follow _nlo_integrand x Jacobian,
bk/derivatives.py:322-335 and 490-612, with the kernels of bk_kernels/k2.py:8-39 and
bk_kernels/kf.py:10-41 in their cancellation-free forms) statement by statement over a
counting number type, and runs it on the workload's sample points.

Counting rules:

* arithmetic = +, -, *, / with at least one operand that varies per sample or per
  (sample, parent) pair; operations on parent-only or constant values are hoisted out of
  the sample loop and not counted; negation, comparisons, fabs, fmin and fmax are not
  counted (selects);
* special = sqrt, exp, log, sin, cos, expm1, log1p (one each);
* the per-sample part (``k2_prepare``: the daughter dipoles z, z', |z - z'|, their three
  amplitudes and the Jacobian) is counted once per sample, the per-pair part (``k2_eval``)
  once per (sample, parent).

``tests/test_census.py`` checks that the restatement returns the C oracle's values and
that the census constants in ``bench.py`` are what ``census()`` returns.

    python -m oracle.census        # prints the census on the headline workload's final state
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


class Tally:
    arithmetic = 0
    special = 0

    @classmethod
    def reset(cls) -> None:
        cls.arithmetic = 0
        cls.special = 0


class V:
    """A float that counts the arithmetic done with it."""

    __slots__ = ("v",)

    def __init__(self, v: float) -> None:
        self.v = float(v)

    @staticmethod
    def _val(x) -> float:
        return x.v if isinstance(x, V) else float(x)

    def _op(self, other, fn):
        Tally.arithmetic += 1
        return V(fn(self.v, V._val(other)))

    def __add__(self, o): return self._op(o, lambda a, b: a + b)
    def __radd__(self, o): return self._op(o, lambda a, b: b + a)
    def __sub__(self, o): return self._op(o, lambda a, b: a - b)
    def __rsub__(self, o): return self._op(o, lambda a, b: b - a)
    def __mul__(self, o): return self._op(o, lambda a, b: a * b)
    def __rmul__(self, o): return self._op(o, lambda a, b: b * a)
    def __truediv__(self, o): return self._op(o, lambda a, b: a / b)
    def __rtruediv__(self, o): return self._op(o, lambda a, b: b / a)
    def __neg__(self): return V(-self.v)
    def __lt__(self, o): return self.v < V._val(o)
    def __le__(self, o): return self.v <= V._val(o)
    def __gt__(self, o): return self.v > V._val(o)
    def __ge__(self, o): return self.v >= V._val(o)
    def __float__(self): return self.v


def _special(fn):
    def wrapped(x):
        if isinstance(x, V):
            Tally.special += 1
            return V(fn(x.v))
        return fn(float(x))
    return wrapped


def _expm1(x: float) -> float:
    return math.expm1(x)


exp, log, sin, cos, sqrt = (_special(f) for f in (math.exp, math.log, math.sin, math.cos, math.sqrt))
expm1, log1p = _special(_expm1), _special(math.log1p)


def fabs(x):
    return V(abs(x.v)) if isinstance(x, V) else abs(x)


def fmin(a, b):
    return a if V._val(a) <= V._val(b) else b


def fmax(a, b):
    return a if V._val(a) >= V._val(b) else b


def isfinite(x) -> bool:
    return math.isfinite(V._val(x))


# --------------------------------------------------------------------------- spline
@dataclass
class Spline:
    x: np.ndarray
    a: np.ndarray
    b: np.ndarray
    c: np.ndarray
    d: np.ndarray
    rmin: float
    rmax: float


def spline_interval(s: Spline, lx) -> int:
    i = int(np.searchsorted(s.x, V._val(lx), side="right")) - 1
    return min(max(i, 0), s.x.size - 2)


def spline_poly(s: Spline, lx):
    i = spline_interval(s, lx)
    dx = lx - float(s.x[i])
    return float(s.a[i]) + dx * (float(s.b[i]) + dx * (float(s.c[i]) + dx * float(s.d[i])))


@dataclass
class NSV:
    p: object
    N: object
    S: object
    edge: int


def eval_s(s: Spline, r) -> NSV:
    if r < s.rmin:
        return NSV(0.0, 0.0, 1.0, -1)
    if r > s.rmax:
        return NSV(0.0, 1.0, 0.0, 1)
    p = spline_poly(s, log(r))
    S = exp(p)
    if not isfinite(S):
        return NSV(p, 1.0, 0.0, 1)
    return NSV(p, -expm1(p), S, 0)


def ndiff_s(A: NSV, B: NSV):
    if A.edge == 0 and B.edge == 0:
        return A.S * expm1(B.p - A.p)
    if V._val(A.N) < 0.5 and V._val(B.N) < 0.5:
        return A.N - B.N
    return B.S - A.S


# --------------------------------------------------------------------------- coupling
@dataclass
class Physics:
    nc: float = 3.0
    nf: float = 3.0
    lambda_qcd: float = 0.241
    c2: float = 1.0
    symmetrize: bool = True


def alpha_smooth(log_d, p: Physics):
    b0 = (11.0 * p.nc - 2.0 * p.nf) / (12.0 * math.pi)
    c = 0.2
    left = 2.0 / c * math.log(2.5)
    log_scale = math.log(4.0 * p.c2 / (p.lambda_qcd * p.lambda_qcd)) - 2.0 * log_d
    right = log_scale / c
    m = fmax(left, right)
    lae = m + log1p(exp(-fabs(left - right)))
    return 1.0 / ((b0 * c) * lae)


# --------------------------------------------------------------------------- kernels
def nlo_kernels_stable(r: float, z, z2, c1, c2, c12, Xsq, X2sq, zzsq, nf_over_nc):
    a = Xsq * z2 * z2
    b = X2sq * z * z
    s = a + b
    dd = r * (r * (z2 * z2 - z * z) - 2.0 * z * z2 * (z2 * c1 - z * c2))
    t = dd / s
    if V._val(fabs(t)) < 0.1:
        t2 = t * t
        series = 0.0
        for k in range(12, 0, -1):
            series = series * t2 + 1.0 / (2.0 * k + 1.0)
        hm1 = t2 * series
        Ld = 2.0 * t * (1.0 + hm1)
    else:
        Ld = log(a / b)
        hm1 = Ld / (2.0 * t) - 1.0
    L = 2.0 * (1.0 + hm1) / s
    f = 2.0 * hm1
    q = 1.0 / zzsq
    r2 = r * r
    C0 = f * q * q - 4.0 * r2 * L * q
    B1 = r * z2 - r * z * c12 - z * z2 * c1 + z * z * c2
    B2 = r * z - r * z2 * c12 - z * z2 * c2 + z2 * z2 * c1
    k2 = C0 + L * r2 * q * 2.0 * r * B1 / (Xsq * z2)
    k2s = C0 + L * r2 * q * 2.0 * r * B2 / (X2sq * z)
    kf = (r2 * L * q - f * q * q) * nf_over_nc
    return k2, k2s, kf


@dataclass
class Point:
    z: object
    z2: object
    c1: object
    c2: object
    c12: object
    s1: object
    s2: object
    zzsq: object
    log_min_pt: object
    Y: NSV
    Y2: NSV
    zz: NSV
    dN: object
    jac: object
    invalid: bool


def k2_prepare(lz, lz2, th, th2, sspl: Spline) -> Point:
    lz, lz2, th, th2 = V(lz), V(lz2), V(th), V(th2)
    z = exp(lz)
    z2 = exp(lz2)
    s1, s2, s12 = sin(0.5 * th), sin(0.5 * th2), sin(0.5 * (th - th2))
    c1, c2, c12 = cos(th), cos(th2), cos(th - th2)
    zzsq = (z - z2) * (z - z2) + 4.0 * z * z2 * s12 * s12
    invalid = V._val(zzsq) < 1e-40 or V._val(z) < 1e-20 or V._val(z2) < 1e-20
    zz = sqrt(zzsq)
    log_min_pt = fmin(fmin(lz, lz2), 0.5 * log(zzsq))
    Y, Y2, ZZ = eval_s(sspl, z), eval_s(sspl, z2), eval_s(sspl, zz)
    return Point(z, z2, c1, c2, c12, s1 * s1, s2 * s2, zzsq, log_min_pt, Y, Y2, ZZ, ndiff_s(Y2, Y),
                 exp(2.0 * lz + 2.0 * lz2), invalid)


def k2_eval(r: float, log_r: float, pt: Point, sspl: Spline, p: Physics):
    if pt.invalid:
        return 0.0, 0.0
    z, z2 = pt.z, pt.z2
    Xsq = (r - z) * (r - z) + 4.0 * r * z * pt.s1
    X2sq = (r - z2) * (r - z2) + 4.0 * r * z2 * pt.s2
    if V._val(Xsq) < 1e-40 or V._val(X2sq) < 1e-40:
        return 0.0, 0.0
    vX, vX2 = eval_s(sspl, sqrt(Xsq)), eval_s(sspl, sqrt(X2sq))
    k2, k2s, kf = nlo_kernels_stable(r, z, z2, pt.c1, pt.c2, pt.c12, Xsq, X2sq, pt.zzsq, p.nf / p.nc)
    dip = vX.S * (pt.Y.S * pt.zz.N + pt.zz.S * pt.dN)
    dips = vX2.S * (pt.Y2.S * pt.zz.N - pt.zz.S * pt.dN)
    if V._val(fabs(k2)) > 1e10 and V._val(fabs(dip)) < 1e-10:
        k2, dip = 0.0, 0.0
    if V._val(fabs(k2s)) > 1e10 and V._val(fabs(dips)) < 1e-10:
        k2s, dips = 0.0, 0.0
    k2res = 0.5 * (k2 * dip + k2s * dips) if p.symmetrize else k2 * dip
    kfres = 0.0
    if p.nf > 0.0:
        dNX = ndiff_s(vX, vX2)
        fermion = 0.5 * kf * dNX * pt.dN if p.symmetrize else kf * pt.Y.S * dNX
        kfres = -fermion
    log_min = fmin(fmin(log_r, pt.log_min_pt), 0.5 * fmin(log(Xsq), log(X2sq)))
    alpha = alpha_smooth(log_min, p)
    scale = (alpha * p.nc) * (alpha * p.nc) / (8.0 * math.pi ** 4) * pt.jac
    return k2res * scale, kfres * scale


def integrand(r: float, x, sspl: Spline, p: Physics) -> tuple[float, float]:
    """_nlo_integrand x Jacobian at x = (log z, log z', theta_z, theta_z')."""
    pt = k2_prepare(x[0], x[1], x[2], x[3], sspl)
    k2, kf = k2_eval(r, math.log(r), pt, sspl, p)
    return V._val(k2), V._val(kf)


# --------------------------------------------------------------------------- census
def census(N: np.ndarray, r: np.ndarray, samples: int = 96, parent_stride: int = 4) -> dict:
    """Mean arithmetic and special operations per sample (k2_prepare) and per (sample,
    parent) pair (k2_eval), over the first `samples` Sobol points of the workload's box and
    every `parent_stride`-th active parent of the amplitude row N."""
    import oracle

    sp = oracle.loglog_spline(r, N, 1)
    sspl = Spline(sp.x, sp.a, sp.b, sp.c, sp.d, sp.rmin, sp.rmax)
    phys = Physics()
    lower, width = oracle.nlo_box(r)
    state, shift = oracle.sobol_state(4, 0)
    u = oracle.sobol(state, shift, 0, samples, as_f32=False)
    x = lower + width * u
    active = np.nonzero((np.arange(r.size) > 0) & (N <= 0.99999))[0][::parent_stride]
    Tally.reset()
    points = [k2_prepare(*row, sspl) for row in x]
    sample_ar, sample_sp = Tally.arithmetic / samples, Tally.special / samples
    Tally.reset()
    for i in active:
        rr = float(r[i])
        lr = math.log(rr)
        for pt in points:
            k2_eval(rr, lr, pt, sspl, phys)
    pairs = samples * active.size
    return {"eval_arithmetic": Tally.arithmetic / pairs, "eval_special": Tally.special / pairs,
            "sample_arithmetic": sample_ar, "sample_special": sample_sp, "samples": samples,
            "parents": int(active.size)}


def workload_census() -> dict:
    """The census on the headline workload's final state (the oracle's evolution rows at
    Y = 10, oracle/evolution_rows_400r.npz), rounded to whole operations."""
    from pathlib import Path

    with np.load(Path(__file__).resolve().parent / "evolution_rows_400r.npz") as data:
        r, N = data["r"], data["N"][-1]
    c = census(N, r)
    return {k: int(round(c[k])) for k in ("eval_arithmetic", "eval_special", "sample_arithmetic", "sample_special")}


if __name__ == "__main__":
    print(workload_census())
