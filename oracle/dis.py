"""CPU FP64 oracle for the NLO DIS integrands -- TEST INFRASTRUCTURE ONLY.

The checker for the device DIS path: ``tests/`` import it to compute reference
values on the same points the CUDA kernels consume.  The product package
``nlo_bk_optimized_b200`` never imports it.

A numpy restatement (vectorised over sample points, float64) of the reference
``torch_nlo_clean/src/nlo_torch`` DIS path.  Map to the reference:

* couplings ``alpha_freeze`` / ``alpha_smooth``    -- coupling.py:49-97
* ``gbw``                                          -- dipole/amplitude.py:23-45
* ``TableDipole`` (local and initialised splines)  -- dipole/amplitude.py:48-252,
                                                      numerics/interpolation.py:10-77
* ``lo_integrand``                                 -- dis/lo.py:12-51, dis/observables.py:352-359
* dipole terms T0/T1/T2 and Omega_L/ab/cd          -- dis/transverse.py:13-300,
                                                      dis/longitudinal.py:12-156
* ``dip_integrand`` (unit-cube map)                -- dis/observables.py:107-172
* qg I1 (dipole UV subtraction + tripole)          -- dis/transverse.py:302-560,
                                                      dis/longitudinal.py:159-214
* qg I2 / I3 and the G functions                   -- dis/transverse.py:341-369, 565-1033,
                                                      dis/longitudinal.py:217-334
* ``qg_integrand`` (unit-cube map)                 -- dis/observables.py:175-250
* nested I2/I3 inner rule (y = t^3, 48 nodes)       -- custom_kernels/dis/i2_i3/extension.py:21-35
                                                      with dis/observables.py:253-331
* ``vegas_iteration`` / ``adapt_edges``            -- numerics/integration.py:120-589, 804-866
* ``gauss_legendre_tensor``                        -- numerics/integration.py:94-117, 749-801
* result scaling (sigma, F_T, F_L, F_2)            -- dis/observables.py:334-624

Bessel functions come from scipy.special (K0, K1), the dilogarithm from
scipy.special.spence (Li2(x) = spence(1 - x)); the reference calls torch.special
and its own series (numerics/special.py:10-96).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
from scipy import special

ALPHA_EM = 1 / 137.035999
NC = 3.0
CF = (NC * NC - 1) / (2 * NC)
LAMBDA_QCD = 0.241
Q0SQR = 1.0
ZMIN = 1e-6
EULER_GAMMA = 0.5772156649015329
E_GAMMA = math.exp(EULER_GAMMA)
PI2_6 = math.pi**2 / 6


# ----------------------------------------------------------------------------- special functions


def k0(x):
    return special.k0(x)


def k1(x):
    return special.k1(x)


def k2(x):
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(x == 0, np.inf, special.k0(x) + 2 * special.k1(x) / np.where(x == 0, 1, x))


def li2(x):
    """Li2(x) = spence(1 - x); below |x| = 0.05 the power series sum x^k / k^2, where
    forming 1 - x would round away the argument."""
    x = np.asarray(x, dtype=np.float64)
    series = np.zeros_like(x)
    term = np.ones_like(x)
    for k in range(1, 25):
        term = term * x
        series = series + term / (k * k)
    return np.where(np.abs(x) < 0.05, series, special.spence(1 - x))


# ----------------------------------------------------------------------------- configuration


@dataclass(frozen=True)
class Kinematics:
    """One (Q^2, x_Bj) point, one quark and the DIS switches that the integrands read."""

    Q2: float
    xbj: float
    mf: float
    transverse: bool = True
    maxr: float = 30.0
    finite_nc: bool = True
    parent_coupling: bool = False  # RunningCouplingScheme.PARENT (else SMALLEST)
    smooth_coupling: bool = False  # RunningCouplingIRScheme.SMOOTH (else FREEZE)
    c2_alpha: float = 1.0
    active_flavors: int = 4
    max_alpha: float = 0.7
    mass_dependent_x: bool = False  # HeavyQuarkX.MassDependentX


def alpha_freeze(r, nf, c2=1.0, max_alpha=0.7):
    b0 = (11 * NC - 2 * nf) / (12 * math.pi)
    arg = 4 * c2 / (r * r * LAMBDA_QCD**2)
    with np.errstate(divide="ignore", invalid="ignore"):
        a = 1 / (b0 * np.log(arg))
    return np.where((a > max_alpha) | (arg < 1), max_alpha, a)


def alpha_smooth(r, nf, c2=1.0):
    b0 = (11 * NC - 2 * nf) / (12 * math.pi)
    c = 0.2
    first = 2 / c * math.log(2.5)
    second = np.log(4 * c2 / (r * r * LAMBDA_QCD**2)) / c
    return 1 / (b0 * c * np.logaddexp(first, second))


def alpha_bar(r, kin: Kinematics):
    a = (alpha_smooth(r, kin.active_flavors, kin.c2_alpha) if kin.smooth_coupling
         else alpha_freeze(r, kin.active_flavors, kin.c2_alpha, kin.max_alpha))
    return a * CF / math.pi


# ----------------------------------------------------------------------------- dipole amplitudes


@dataclass(frozen=True)
class GBWDipole:
    qs0sqr: float = 0.1
    lam: float = 0.3
    gamma: float = 1.0
    x0: float = 1.0
    min_r: float = 1e-30
    max_r: float = 1e3

    def X0(self) -> float:
        return self.x0

    def __call__(self, r, Y):
        y0 = math.log(1 / self.x0)
        qs2 = self.qs0sqr * np.exp(self.lam * np.maximum(Y, y0))
        arg = np.power(r * r * qs2, self.gamma) / 4
        return np.where(np.abs(arg) < 1e-7, arg, 1 - np.exp(-arg))


def natural_spline_second_derivatives(x, y):
    """Second derivatives of the natural cubic spline through (x, y) along the last axis
    (numerics/interpolation.py:28-40): zero at both ends, interior by the tridiagonal solve."""
    h = np.diff(x, axis=-1)
    n = x.shape[-1]
    diag = 2 * (h[..., :-1] + h[..., 1:])
    rhs = 6 * ((y[..., 2:] - y[..., 1:-1]) / h[..., 1:] - (y[..., 1:-1] - y[..., :-2]) / h[..., :-1])
    m = n - 2
    c = np.zeros_like(diag)
    d = np.zeros_like(rhs)
    c[..., 0] = h[..., 1] / diag[..., 0] if m > 1 else 0
    d[..., 0] = rhs[..., 0] / diag[..., 0]
    for i in range(1, m):
        off = h[..., i]
        den = diag[..., i] - off * c[..., i - 1]
        if i < m - 1:
            c[..., i] = h[..., i + 1] / den
        d[..., i] = (rhs[..., i] - off * d[..., i - 1]) / den
    sol = np.zeros_like(d)
    sol[..., m - 1] = d[..., m - 1]
    for i in range(m - 2, -1, -1):
        sol[..., i] = d[..., i] - c[..., i] * sol[..., i + 1]
    zeros = np.zeros((*y.shape[:-1], 1))
    return np.concatenate((zeros, sol, zeros), axis=-1)


def spline_eval(x, y, M, xe, interval):
    """Evaluate the natural spline (x, y, second derivatives M) at xe in `interval`
    with the power form a + dx (b + dx (c + dx d)) of numerics/interpolation.py:42-77."""
    def take(arr, idx):
        return arr[idx] if arr.ndim == 1 else np.take_along_axis(arr, idx[..., None], axis=-1)[..., 0]

    x0 = take(x, interval)
    x1 = take(x, interval + 1)
    y0 = take(y, interval)
    y1 = take(y, interval + 1)
    m0 = take(M, interval)
    m1 = take(M, interval + 1)
    h = x1 - x0
    b = (y1 - y0) / h - h * (2 * m0 + m1) / 6
    c = m0 / 2
    d = (m1 - m0) / (6 * h)
    dx = xe - x0
    return y0 + dx * (b + dx * (c + dx * d))


class TableDipole:
    """BK-table dipole N(r, Y) of dipole/amplitude.py:48-252; ``interpolation`` is
    "spline_linear" (the default) or "linear_linear" (bilinear in r and Y, :188-212)."""

    def __init__(self, r, y, N, x0=1.0, interpolation="spline_linear"):
        if interpolation not in ("spline_linear", "linear_linear"):
            raise ValueError("interpolation is 'spline_linear' or 'linear_linear'")
        self.interpolation = interpolation
        self.r = np.asarray(r, dtype=np.float64)
        self.Y = np.asarray(y, dtype=np.float64) + max(0.0, math.log(1 / x0))
        self.N = np.asarray(N, dtype=np.float64)
        self.min_r = float(self.r[0])
        self.max_r = float(self.r[-1])
        self.init_Y = -1.0
        self.init_M = None
        self.init_N = None
        self.maxr_interpolate = -1.0

    def X0(self) -> float:
        return 1.0

    def local(self, r, Y):
        """7-point (9 at the top) natural spline in r of the Y-interpolated rows."""
        r = np.asarray(r, dtype=np.float64)
        Y = np.asarray(Y, dtype=np.float64)
        nr = self.r.size
        rind = np.searchsorted(self.r, r, side="right") - 1
        yind = np.searchsorted(self.Y, Y, side="right") - 1
        yind2 = np.minimum(yind + 1, self.Y.size - 1)
        dY = np.where(yind2 != yind, self.Y[yind2] - self.Y[yind], 1.0)
        frac = np.where(yind2 != yind, (Y - self.Y[yind]) / dY, 0.0)
        out = np.empty_like(r)
        upper = rind + 3 > nr - 1
        for points, mask in ((7, ~upper), (9, upper)):
            if not mask.any():
                continue
            if points == 7:
                start = np.maximum(rind[mask] - 3, 0)
            else:
                start = np.full(mask.sum(), nr - 9)
            idx = start[:, None] + np.arange(points)
            lo = self.N[yind[mask][:, None], idx]
            hi = self.N[yind2[mask][:, None], idx]
            vals = lo + frac[mask][:, None] * (hi - lo)
            xs = self.r[idx]
            M = natural_spline_second_derivatives(xs, vals)
            interval = np.clip(rind[mask] - start, 0, points - 2)
            out[mask] = spline_eval(xs, vals, M, r[mask], interval)
        return out

    def bilinear(self, r, Y):
        """LINEAR_LINEAR amplitude (dipole/amplitude.py:188-212): bilinear in (r, Y) with the
        same expression order; the last Y row interpolates in r only; r on the last knot
        gives 1."""
        r = np.asarray(r, dtype=np.float64)
        Y = np.asarray(Y, dtype=np.float64)
        nr, ny = self.r.size, self.Y.size
        rind = np.searchsorted(self.r, r, side="right") - 1
        yind = np.searchsorted(self.Y, Y, side="right") - 1
        rind2 = np.minimum(rind + 1, nr - 1)
        yind2 = np.minimum(yind + 1, ny - 1)
        r1, r2 = self.r[rind], self.r[rind2]
        Y1, Y2 = self.Y[yind], self.Y[yind2]
        dr = np.where(rind2 != rind, r2 - r1, 1.0)
        dY = np.where(yind2 != yind, Y2 - Y1, 1.0)
        N11 = self.N[yind, rind]
        N12 = self.N[yind, rind2]
        N21 = self.N[yind2, rind]
        N22 = self.N[yind2, rind2]
        value = (N11 * (r2 - r) * (Y2 - Y) + N12 * (r - r1) * (Y2 - Y)
                 + N21 * (r2 - r) * (Y - Y1) + N22 * (r - r1) * (Y - Y1)) / (dr * dY)
        last_Y = N11 + (r - r1) / dr * (N12 - N11)
        value = np.where(yind2 == yind, last_Y, value)
        return np.where(rind2 == rind, 1.0, value)

    def _clamped(self, r, Y):
        r = np.where(r < self.min_r, self.min_r * 1.000001, r)
        r = np.where(r > self.max_r, self.max_r * 0.999999, r)
        Y = np.where((Y >= 0) & (Y < self.Y[0]), self.Y[0], Y)
        if np.any((Y < self.Y[0]) | (Y > self.Y[-1])):
            raise ValueError("Y outside the table")
        return r, Y

    def initialized(self, Y):
        Y = np.asarray(Y, dtype=np.float64)
        near_zero = (np.abs(Y) < 0.001) & (abs(self.init_Y) < 0.001)
        den = np.minimum(Y, self.init_Y)
        safe = np.where(den != 0, den, 1.0)
        match = (self.init_Y >= 0) & (np.abs(Y - self.init_Y) / safe < 0.001)
        return (near_zero | match) & (self.init_M is not None)

    def initialize(self, Y):
        """initialize_interpolation (dipole/amplitude.py:105-133) and the maxr search (:254-272)."""
        Y = float(Y)
        if 0 <= Y <= self.Y[0]:
            Y = float(self.Y[0])
        if Y < 0 or Y > self.Y[-1]:
            raise ValueError("cannot initialise outside the table")
        if self.init_M is not None and bool(self.initialized(np.array(Y))):
            return
        self.init_M = None
        self.init_Y = -1.0
        self.maxr_interpolate = -1.0
        er = self.r.copy()
        er[0] *= 1.0001
        er[-1] *= 0.9999
        N = self(er, np.full_like(er, Y))
        self.init_N = N
        self.init_M = natural_spline_second_derivatives(self.r, N)
        self.init_Y = Y
        step, previous, r = 2.0, 0.1, 0.01
        for _ in range(41):
            if r > self.max_r:
                break
            v = float(self(np.array([r]), np.array([Y]))[0])
            if v >= 0.99999:
                if step < 1e-2:
                    self.maxr_interpolate = r
                    return
                step /= 1.5
                r = previous
            previous = r
            r += step
        self.maxr_interpolate = -1.0

    def global_spline(self, r):
        interval = np.clip(np.searchsorted(self.r, r, side="right") - 1, 0, self.r.size - 2)
        v = spline_eval(self.r, self.init_N, self.init_M, r, interval)
        if self.maxr_interpolate > 0:
            v = np.where(r >= self.maxr_interpolate, 1.0, v)
        return np.clip(v, 0, 1)

    def __call__(self, r, Y):
        r, Y = np.broadcast_arrays(np.asarray(r, dtype=np.float64), np.asarray(Y, dtype=np.float64))
        r, Y = self._clamped(r, Y)
        init = self.initialized(Y)
        out = np.empty_like(r)
        if init.any():
            out[init] = self.global_spline(r[init])
        if (~init).any():
            plain = self.bilinear if self.interpolation == "linear_linear" else self.local
            out[~init] = np.clip(plain(r[~init], Y[~init]), 0, 1)
        return out


# ----------------------------------------------------------------------------- LO


def lo_psi2(r, z, Q2, quarks, transverse):
    """sum_q e_q^2 |Psi|^2 without N and Jacobian (dis/lo.py:22-49); quarks = [(mass, e^2)]."""
    total = np.zeros_like(r)
    for mf, e2 in quarks:
        eps = np.sqrt(Q2 * z * (1 - z) + mf * mf)
        arg = r * eps
        active = (arg >= 1e-7) & (arg <= 5e2)
        a = np.where(active, arg, 1.0)
        if transverse:
            v = e2 * ((1 - 2 * z + 2 * z * z) * eps * eps * k1(a) ** 2 + (mf * k0(a)) ** 2)
        else:
            v = e2 * 4 * Q2 * z * z * (1 - z) ** 2 * k0(a) ** 2
        total = total + np.where(active, v, 0.0)
    return total


def lo_integrand(x, Q2, xbj, quarks, transverse, dipole, maxr=30.0):
    """Unit-square LO integrand with the 2 pi r maxr Jacobian (dis/observables.py:352-359)."""
    z = x[:, 0]
    r = maxr * x[:, 1]
    Y = max(math.log(dipole.X0() / xbj), 0.0)
    return 2 * math.pi * r * maxr * lo_psi2(r, z, Q2, quarks, transverse) * dipole(r, np.full_like(r, Y))


# ----------------------------------------------------------------------------- dipole (virtual) terms


def _gamma_m(Q2, mf):
    return math.sqrt(1 + 4 * mf * mf / Q2)


def _log_mass_ratio(z, Q2, mf):
    return np.log((z * (1 - z) * Q2 + mf * mf) / (mf * mf))


def _omega_t_core(z, gam):
    return np.log(1 - z) + gam * np.log((1 + gam) / (1 + gam - 2 * z))


def omega_t_v(Q2, z, mf):
    gam = _gamma_m(Q2, mf)
    m2q = mf * mf / Q2

    def half(zz):
        return ((1 + 1 / (2 * zz)) * _omega_t_core(zz, gam)
                - 1 / (2 * zz) * ((zz + 0.5) * (1 - gam) + m2q) * _log_mass_ratio(zz, Q2, mf))

    return half(z) + half(1 - z)


def omega_t_n(Q2, z, mf):
    gam = _gamma_m(Q2, mf)
    m2q = mf * mf / Q2

    def half(zz):
        return ((1 + zz - 2 * zz * zz) / zz * _omega_t_core(zz, gam)
                + (1 - zz) / zz * ((0.5 + zz) * (gam - 1) - m2q) * _log_mass_ratio(zz, Q2, mf))

    return half(z) - half(1 - z)


def omega_l_v(Q2, z, mf):
    gam = _gamma_m(Q2, mf)
    return (1 / (2 * z) * _omega_t_core(z, gam)
            + 1 / (2 * (1 - z)) * _omega_t_core(1 - z, gam)
            + 1 / (4 * z * (1 - z)) * (gam - 1 + 2 * mf * mf / Q2) * _log_mass_ratio(z, Q2, mf))


def l_dip(Q2, z, mf):
    gam = _gamma_m(Q2, mf)
    total = 0.0
    for zz in (z, 1 - z):
        total = total + li2(1 / (1 - (1 - gam) / (2 * zz))) + li2(1 / (1 - (1 + gam) / (2 * zz)))
    return total - (PI2_6 - 0.5 * np.log(z / (1 - z)) ** 2)


def _kappa(z, Q2, mf):
    return np.sqrt(z * (1 - z) * Q2 + mf * mf)


def t_dip0(Q2, z, r2, mf):
    r = np.sqrt(r2)
    kz = _kappa(z, Q2, mf)
    common = -PI2_6 + 0.5 * np.log(z / (1 - z)) ** 2 + omega_t_v(Q2, z, mf) + l_dip(Q2, z, mf)
    t1 = (kz * k1(r * kz)) ** 2 * ((z * z + (1 - z) ** 2) * (2.5 + common)
                                   + (2 * z - 1) / 2 * omega_t_n(Q2, z, mf))
    t2 = (mf * k0(r * kz)) ** 2 * (3 + common)
    return t1 + t2


def _xi_factor(xi):
    return 1 / xi * (2 * np.log(xi) / (1 - xi) - (1 + xi) / 2)


def t_dip1(Q2, z, r2, mf, xi):
    r = np.sqrt(r2)
    kz = _kappa(z, Q2, mf)
    v1 = 0.0
    vms1 = 0.0
    for zz in (z, 1 - z):
        sh = np.sqrt(kz * kz + xi / (1 - xi) * (1 - zz) * mf * mf)
        k1s = k1(r * sh)
        diff = sh * k1s - kz * k1(r * kz)
        v1 = v1 + _xi_factor(xi) * diff - (np.log(xi) / (1 - xi) ** 2 + zz / (1 - xi) + zz / 2) * (
            1 - zz) * mf * mf / sh * k1s
        k0s = k0(r * sh)
        vms1 = vms1 + _xi_factor(xi) * (k0s - k0(r * kz)) + (-1.5 * (1 - zz) / (1 - xi) + (1 - zz) / 2) * k0s
    return kz * k1(r * kz) * (z * z + (1 - z) ** 2) * v1 + mf * mf * k0(r * kz) * vms1


def weighted_k1_difference(r, kb, delta):
    """sqrt(kb^2 + delta) K1(r sqrt(.)) - kb K1(r kb), linearised below 1e-5 relative
    (dis/transverse.py:13-23)."""
    base2 = kb * kb
    shifted2 = base2 + delta
    valid = (shifted2 > 0) & (kb > 0)
    rel = np.abs(delta) / (base2 + np.abs(delta) + 1e-300)
    linear = -0.5 * r * delta * k0(r * kb)
    sh = np.sqrt(np.maximum(shifted2, 0))
    direct = sh * k1(r * sh) - kb * k1(r * kb)
    return np.where(valid, np.where(rel < 1e-5, linear, direct), 0.0)


def _t2_side(Q2, zz, mf, r, ychi, yu):
    """(V2, VMS2, N) unsymmetric pieces at momentum fraction zz (dis/transverse.py:168-300)."""
    m2 = mf * mf
    chi = zz * ychi
    u = (1 - yu) / yu
    kz = _kappa(zz, Q2, mf)
    kc2 = chi * (1 - chi) * Q2 + m2
    delta = u * (1 - zz) / (1 - chi) * kc2
    sh = np.sqrt(kz * kz + delta)
    k1s = k1(r * sh)
    k0s = k0(r * sh)
    uu = u / (u + 1)
    pre = zz / (yu * yu)
    v2 = pre * (
        -1 / (1 - chi) / (u * (u + 1)) * m2 / kc2
        * (2 * chi + uu * uu / zz * (zz - chi) * (1 - 2 * chi)) * weighted_k1_difference(r, kz, delta)
        - 1 / (1 - chi) ** 2 / (u + 1) * (zz - chi)
        * (1 - 2 * uu * (zz - chi) + uu * uu / zz * (zz - chi) ** 2) * m2 / sh * k1s)
    vms2 = pre * (
        1 / (1 - chi) / (u + 1) ** 2 * (-zz - uu * (zz + u * chi) / zz * (chi - (1 - zz))) * k0s
        + 1 / (u + 1) ** 3 * (kz * kz / kc2 * (1 + u * chi * (1 - chi) / (zz * (1 - zz)))
                              - m2 / kc2 * chi / (1 - chi)
                              * (2 * (1 + u) ** 2 / u + u / (zz * (1 - zz)) * (zz - chi) ** 2))
        * (k0s - k0(r * kz)))
    pref = 2 * (1 - zz) / zz / (u + 1) ** 3
    n = pre * (pref * ((2 + u) * u * zz + u * u * chi) * sh * k1s
               + pref * m2 / kc2 * (zz / (1 - zz) + chi / (1 - chi) * (u - 2 * zz - 2 * u * chi))
               * (sh * k1s - kz * k1(r * kz)))
    return v2, vms2, n


def t_dip2(Q2, z, r2, mf, ychi, yu):
    r = np.sqrt(r2)
    kz = _kappa(z, Q2, mf)
    a = _t2_side(Q2, z, mf, r, ychi, yu)
    b = _t2_side(Q2, 1 - z, mf, r, ychi, yu)
    v2 = a[0] + b[0]
    vms2 = a[1] + b[1]
    n = a[2] - b[2]
    return (kz * k1(r * kz) * ((z * z + (1 - z) ** 2) * v2 + (2 * z - 1) / 2 * n)
            + mf * mf * k0(r * kz) * vms2)


def l_omega_const(Q2, z, r, mf):
    ff = 4 * Q2 * (z * (1 - z)) ** 2
    arg = np.sqrt(Q2 * z * (1 - z) + mf * mf) * r
    active = arg >= 1e-7
    a = np.where(active, arg, 1.0)
    v = ff * k0(a) ** 2 * (2.5 - PI2_6 + 0.5 * np.log(z / (1 - z)) ** 2
                           + omega_l_v(Q2, z, mf) + l_dip(Q2, z, mf))
    return np.where(active, v, 0.0)


def l_ab(Q2, z, r, mf, xi):
    ff = 4 * Q2 * (z * (1 - z)) ** 2
    kz = _kappa(z, Q2, mf)
    m2 = mf * mf
    b1 = k0(kz * r)
    b2 = k0(np.sqrt(kz * kz + (1 - z) * xi / (1 - xi) * m2) * r)
    b3 = k0(np.sqrt(kz * kz + z * xi / (1 - xi) * m2) * r)
    return ff * b1 / xi * (-2 * np.log(xi) / (1 - xi) + (1 + xi) / 2) * (2 * b1 - b2 - b3)


def l_cd(Q2, z, r, mf, xi, x):
    ff = 4 * Q2 * (z * (1 - z)) ** 2
    kz = _kappa(z, Q2, mf)
    kz2 = kz * kz
    m2 = mf * mf
    arg = kz * r
    active = arg >= 1e-7
    b1 = k0(np.where(active, arg, 1.0))
    total = 0.0
    for za, zb in ((z, 1 - z), (1 - z, z)):
        # za plays z1 in the first term (CLm1, kappa1) and 1 - z1 in the second (CLm2, kappa2)
        den = x * (1 - xi) + xi / zb
        clm = za * za * (1 - xi) / zb * (-xi * xi + x * (1 - xi) * (1 + (1 - xi) * (1 + za * xi / zb)) / den)
        kap = xi * m2 / ((1 - xi) * (1 - x) * den) * (xi * (1 - x) + x * (1 - za * (1 - xi) / zb))
        total = total + (b1 - k0(r * np.sqrt(kz2 / (1 - x) + kap))) * clm / (
            (1 - xi) * (1 - x) * den * (x / (1 - x) * kz2 + kap))
    return ff * np.where(active, b1 * m2 * total, 0.0)


def dipole_rapidity(Q2, xbj, mf, mass_dependent_x):
    W2 = (1 - xbj) * Q2 / xbj
    X = (Q2 + 4 * mf * mf) / (Q2 + W2) if mass_dependent_x else Q2 / (Q2 + W2)
    return math.log(1 / X)


DIP_TERMS = {("T", 0): 2, ("T", 1): 3, ("T", 2): 4, ("L", 0): 2, ("L", 1): 3, ("L", 2): 4}


def dip_integrand(x, kin: Kinematics, order: int, dipole):
    """integrand_dip_massive (dis/observables.py:107-172); order 0/1/2 = T0/T1/T2 or
    Omega_L_const/ab/cd."""
    z1 = ZMIN + x[:, 0] * (1 - 2 * ZMIN)
    x01 = kin.maxr * x[:, 1]
    inside = (x01 >= dipole.min_r) & (x01 <= dipole.max_r)
    r = np.clip(x01, dipole.min_r, dipole.max_r)
    Y = dipole_rapidity(kin.Q2, kin.xbj, kin.mf, kin.mass_dependent_x)
    N01 = dipole(r, np.full_like(r, Y))
    Q2, mf = kin.Q2, kin.mf
    with np.errstate(all="ignore"):
        if kin.transverse:
            v = (t_dip0(Q2, z1, r * r, mf) if order == 0 else
                 t_dip1(Q2, z1, r * r, mf, x[:, 2]) if order == 1 else
                 t_dip2(Q2, z1, r * r, mf, x[:, 2], x[:, 3]))
        else:
            v = (l_omega_const(Q2, z1, r, mf) if order == 0 else
                 l_ab(Q2, z1, r, mf, x[:, 2]) if order == 1 else
                 l_cd(Q2, z1, r, mf, x[:, 2], x[:, 3]))
        out = N01 * v * (x01 * kin.maxr * (1 - 2 * ZMIN)) * alpha_bar(r, kin)
    return np.where(inside & np.isfinite(out), out, 0.0)


# ----------------------------------------------------------------------------- qqbar-g terms


@dataclass
class Tripole:
    """Tripole geometry (dis/transverse.py:937-1000); side 'j' pairs the gluon with quark 0
    (transverse labels; the longitudinal code calls it 'k'), side 'k' with antiquark 1."""

    z0: np.ndarray
    z1: np.ndarray
    z2: np.ndarray
    x20x21: np.ndarray
    Qb2: tuple
    omega: tuple
    lam: tuple
    x2sq: tuple
    x3sq: tuple
    x2jx3j: np.ndarray
    x2kx3k: np.ndarray
    x2jx3k: np.ndarray
    x2kx3j: np.ndarray
    x3jx3k: np.ndarray


def tripole(Q2, z1, z2, x01sq, x02sq, x21sq):
    z0 = 1 - z1 - z2
    x20x21 = -0.5 * (x01sq - x21sq - x02sq)
    fj = z0 / (z0 + z2)
    fk = z1 / (z1 + z2)
    return Tripole(
        z0=z0, z1=z1, z2=z2, x20x21=x20x21,
        Qb2=(Q2 * z1 * (1 - z1), Q2 * z0 * (1 - z0)),
        omega=(z0 * z2 / (z1 * (z0 + z2) ** 2), z1 * z2 / (z0 * (z1 + z2) ** 2)),
        lam=(z1 * z2 / z0, z0 * z2 / z1),
        x2sq=(x02sq, x21sq),
        x3sq=(fj * fj * x02sq + x21sq - 2 * fj * x20x21, fk * fk * x21sq + x02sq - 2 * fk * x20x21),
        x2jx3j=x20x21 - fj * x02sq,
        x2kx3k=-x20x21 + fk * x21sq,
        x2jx3k=-x02sq + fk * x20x21,
        x2kx3j=x21sq - fj * x20x21,
        x3jx3k=fj * x02sq + fk * x21sq - (1 + fj * fk) * x20x21,
    )


def _side_weights(t: Tripole):
    """(2 z_a (z_a + z2) + z2^2)/(z_a + z2)^2 and (1 - 2 z_b (1 - z_b)) per side."""
    P = ((2 * t.z0 * (t.z0 + t.z2) + t.z2**2) / (t.z0 + t.z2) ** 2,
         (2 * t.z1 * (t.z1 + t.z2) + t.z2**2) / (t.z1 + t.z2) ** 2)
    A = (1 - 2 * t.z1 * (1 - t.z1), 1 - 2 * t.z0 * (1 - t.z0))
    return P, A


def g_function(a, b, Qb2, mf, x2sq, x3sq, omega, lam, y):
    """G_integrand_simplified (dis/longitudinal.py:303-334)."""
    m2 = mf * mf
    A = y * lam * m2 + Qb2 + m2
    B = y * x3sq + omega * x2sq
    arg = np.sqrt(A * B / y)
    order = a + b - 2
    K = k0(arg) if order == 0 else k1(arg) if order == 1 else k2(arg)
    return y ** (-0.5 * (2 - a + b)) * 2.0 ** (a + b - 1) * omega ** (b - 1) * (A / B) ** (0.5 * (a + b - 2)) * K


def g_bar(a, b, t: Tripole, s, mf, y):
    return (g_function(a, b, t.Qb2[s], mf, t.x2sq[s], t.x3sq[s], t.omega[s], t.lam[s], y)
            - g_function(a, b, t.Qb2[s], mf, t.x2sq[s], t.x3sq[s], t.omega[s], 0.0, y))


def _X2(t: Tripole, s):
    return t.x3sq[s] + t.omega[s] * t.x2sq[s]


def g22_sing(t, s, mf):
    M2 = t.Qb2[s] + mf * mf
    X2 = _X2(t, s)
    return np.sqrt(M2 / X2) * k1(np.sqrt(M2 * X2)) / t.x2sq[s]


def g12_sing(t, s, mf):
    return k0(np.sqrt((t.Qb2[s] + mf * mf) * _X2(t, s))) / t.x2sq[s]


def h_function(t, s, mf):
    M2 = t.Qb2[s] + mf * mf * (1 + t.lam[s])
    X2 = _X2(t, s)
    return 4 * np.sqrt(M2 / X2) * k1(np.sqrt(M2 * X2))


def _f_bracket(t: Tripole):
    """z2 (z0-z1)^2 (x2j.x3j x2k.x3k - x2k.x3j x2j.x3k) - (...)(...) x20.x21 x3j.x3k."""
    z0, z1, z2 = t.z0, t.z1, t.z2
    return (z2 * (z0 - z1) ** 2 * (t.x2jx3j * t.x2kx3k - t.x2kx3j * t.x2jx3k)
            - (z1 * (z0 + z2) + z0 * (z1 + z2)) * (z0 * (z0 + z2) + z1 * (z1 + z2)) * t.x20x21 * t.x3jx3k)


def t_qg_dipole_uvsub(Q2, mf, z1, z2, x01sq, x02sq, x21sq):
    t = tripole(Q2, z1, z2, x01sq, x02sq, x21sq)
    P, A = _side_weights(t)
    total = 0.0
    for s in (0, 1):
        M2 = t.Qb2[s] + mf * mf
        damp = -np.exp(-t.x2sq[s] / (x01sq * E_GAMMA))
        arg = np.sqrt(x01sq * M2)
        total = total + P[s] / t.x2sq[s] * damp * (A[s] * M2 * k1(arg) ** 2 + mf * mf * k0(arg) ** 2)
    return total


def t_qg_tripole_i1(Q2, mf, z1, z2, x01sq, x02sq, x21sq):
    t = tripole(Q2, z1, z2, x01sq, x02sq, x21sq)
    P, A = _side_weights(t)
    z0 = t.z0
    m2 = mf * mf
    jk = 0.0
    for s in (0, 1):
        M2 = t.Qb2[s] + m2
        X2 = _X2(t, s)
        arg = np.sqrt(X2) * np.sqrt(M2)
        jk = jk + P[s] / t.x2sq[s] * (A[s] * M2 * t.x3sq[s] / X2 * k1(arg) ** 2 + m2 * k0(arg) ** 2)
    G22 = (g22_sing(t, 0, mf), g22_sing(t, 1, mf))
    G12 = (g12_sing(t, 0, mf), g12_sing(t, 1, mf))
    H = (h_function(t, 0, mf), h_function(t, 1, mf))
    zj, zk = z0 + z2, z1 + z2
    F = 0.5 * (
        4 / (zj * zk) * _f_bracket(t) * G22[0] * G22[1]
        - zj * z1 * z2 / zk**2 * t.x2jx3j * H[1] * G22[0]
        + zk * z0 * z2 / zj**2 * t.x2kx3k * H[0] * G22[1]
        - z0**2 * z1 * z2 / zj**3 * t.x2jx3j * H[0] * G22[0]
        + z1**2 * z0 * z2 / zk**3 * t.x2kx3k * H[1] * G22[1]
        + (z0 * z2) ** 2 / (8 * zj**4) * H[0] ** 2
        + (z1 * z2) ** 2 / (8 * zk**4) * H[1] ** 2)
    Fm = 0.5 * m2 * (-((2 * z0 + z2) * (2 * z1 + z2) + z2**2) * t.x20x21 * 64 * G12[0] * G12[1] / (32 * zj * zk))
    return jk + F + Fm


def t_moments_at(t: Tripole, mf, y):
    """The eight G values (Gbar22, Gbar12, G21, G11) x (side j, side k) at one y."""
    out = {}
    for s in (0, 1):
        out[("22", s)] = g_bar(2, 2, t, s, mf, y)
        out[("12", s)] = g_bar(1, 2, t, s, mf, y)
        out[("21", s)] = g_function(2, 1, t.Qb2[s], mf, t.x2sq[s], t.x3sq[s], t.omega[s], t.lam[s], y)
        out[("11", s)] = g_function(1, 1, t.Qb2[s], mf, t.x2sq[s], t.x3sq[s], t.omega[s], t.lam[s], y)
    return out


def t_qg_i2(t: Tripole, mf, G):
    """_IT_tripole_I2 (dis/transverse.py:565-735) written over the G values G[(kind, side)]."""
    z0, z1, z2 = t.z0, t.z1, t.z2
    m2 = mf * mf
    zj, zk = z0 + z2, z1 + z2
    P, A = _side_weights(t)
    G22 = (g22_sing(t, 0, mf), g22_sing(t, 1, mf))
    G12 = (g12_sing(t, 0, mf), g12_sing(t, 1, mf))
    H = (h_function(t, 0, mf), h_function(t, 1, mf))
    jk = 0.0
    jkm = 0.0
    for s in (0, 1):
        M2 = t.Qb2[s] + m2
        X2 = _X2(t, s)
        arg = np.sqrt(X2) * np.sqrt(M2)
        jk = jk + P[s] * A[s] * G[("22", s)] * t.x3sq[s] / 8 * np.sqrt(M2 / X2) * k1(arg)
        jkm = jkm + P[s] * G[("12", s)] / 4 * k0(arg)
    F = 0.5 * (
        _f_bracket(t) / (4 * zj * zk) * (G[("22", 1)] * G22[0] + G[("22", 0)] * G22[1])
        - zj * z1 * z2 / (16 * zk**2) * t.x2jx3j * H[1] * G[("22", 0)]
        + zk * z0 * z2 / (16 * zj**2) * t.x2kx3k * H[0] * G[("22", 1)]
        - z0**2 * z1 * z2 / (16 * zj**3) * t.x2jx3j * H[0] * G[("22", 0)]
        + z1**2 * z0 * z2 / (16 * zk**3) * t.x2kx3k * H[1] * G[("22", 1)])
    c2 = (2 * z0 + z2) * (2 * z1 + z2) + z2**2
    Fm = 0.5 * m2 * (
        -z0 * z1 * z2**2 / (2 * zj**3) * t.x2jx3j * G[("21", 0)] * G12[0]
        + z0 * z1 * z2**2 / (2 * zk**3) * t.x2kx3k * G[("21", 1)] * G12[1]
        - c2 * t.x20x21 / (4 * zj * zk) * (G[("12", 1)] * G12[0] + G[("12", 0)] * G12[1])
        - (z0 * z2) ** 2 / (2 * zj * zk**2) * t.x2jx3k * G[("21", 1)] * G12[0]
        + (z1 * z2) ** 2 / (2 * zj**2 * zk) * t.x2kx3j * G[("21", 0)] * G12[1]
        - z0 * z1 * z2**2 / zj**3 * t.x2jx3j * G[("11", 0)] * G22[0]
        + z0 * z1 * z2**2 / zk**3 * t.x2kx3k * G[("11", 1)] * G22[1]
        - zj * z2**2 / zk**2 * t.x2jx3j * G[("11", 1)] * G22[0]
        + zk * z2**2 / zj**2 * t.x2kx3k * G[("11", 0)] * G22[1]
        + z0 * z2**3 / (4 * zj**4) * H[0] * G[("11", 0)]
        + z1 * z2**3 / (4 * zk**4) * H[1] * G[("11", 1)])
    return jk + m2 * jkm + F + Fm


def t_qg_i3(t: Tripole, mf, G1, G2):
    """_IT_tripole_I3 (dis/transverse.py:738-934) with G1 = G(y_t1), G2 = G(y_t2)."""
    z0, z1, z2 = t.z0, t.z1, t.z2
    m2 = mf * mf
    zj, zk = z0 + z2, z1 + z2
    P, A = _side_weights(t)
    jkm = sum(P[s] * t.x2sq[s] / 64 * G1[("12", s)] * G2[("12", s)] for s in (0, 1))
    jk = sum(P[s] * A[s] * t.x3sq[s] * t.x2sq[s] / 256 * G1[("22", s)] * G2[("22", s)] for s in (0, 1))
    F = 0.5 * G1[("22", 0)] * G2[("22", 1)] / (64 * zj * zk) * _f_bracket(t)
    c2 = (2 * z0 + z2) * (2 * z1 + z2) + z2**2
    Fm = 0.5 * m2 * (
        z2**4 / (64 * zj**4) * (4 * z1 * (z1 - 1) + 2) * t.x3sq[0] * G1[("21", 0)] * G2[("21", 0)]
        + z2**4 / (64 * zk**4) * (4 * z0 * (z0 - 1) + 2) * t.x3sq[1] * G1[("21", 1)] * G2[("21", 1)]
        - z0 * z1 * z2**2 / (16 * zj**3) * t.x2jx3j * G1[("12", 0)] * G2[("21", 0)]
        + z0 * z1 * z2**2 / (16 * zk**3) * t.x2kx3k * G1[("12", 1)] * G2[("21", 1)]
        - c2 * t.x20x21 / (32 * zj * zk) * G1[("12", 0)] * G2[("12", 1)]
        + z2**4 / (32 * zj**2 * zk**2) * c2 * t.x3jx3k * G1[("21", 0)] * G2[("21", 1)]
        + m2 / 8 * (z2 / zj) ** 4 * G1[("11", 0)] * G2[("11", 0)]
        + m2 / 8 * (z2 / zk) ** 4 * G1[("11", 1)] * G2[("11", 1)]
        - (z0 * z2) ** 2 / (16 * zj * zk**2) * t.x2jx3k * G1[("12", 0)] * G2[("21", 1)]
        + (z1 * z2) ** 2 / (16 * zk * zj**2) * t.x2kx3j * G1[("12", 1)] * G2[("21", 0)]
        - z0 * z1 * z2**2 / (16 * zj**3) * t.x2jx3j * G1[("11", 0)] * G2[("22", 0)]
        + z0 * z1 * z2**2 / (16 * zk**3) * t.x2kx3k * G1[("11", 1)] * G2[("22", 1)]
        - zj * z2**2 / (16 * zk**2) * t.x2jx3j * G1[("11", 1)] * G2[("22", 0)]
        + zk * z2**2 / (16 * zj**2) * t.x2kx3k * G1[("11", 0)] * G2[("22", 1)])
    return jk + m2 * jkm + F + Fm


def l_qg_tripole_i1(Q2, mf, z1, z2, x01sq, x02sq, x21sq):
    t = tripole(Q2, z1, z2, x01sq, x02sq, x21sq)
    z0 = t.z0
    b = [k0(np.sqrt(t.Qb2[s] + mf * mf) * np.sqrt(_X2(t, s))) for s in (0, 1)]
    return 4 * Q2 * (
        z1**2 * (2 * z0 * (z0 + z2) + z2**2) / x02sq * b[0] ** 2
        + z0**2 * (2 * z1 * (z1 + z2) + z2**2) / x21sq * b[1] ** 2
        - 2 * z0 * z1 * (z0 * (1 - z0) + z1 * (1 - z1)) * t.x20x21 / (x02sq * x21sq) * b[0] * b[1])


def l_qg_dipole_uvsub(Q2, mf, z1, z2, x01sq, x02sq, x21sq):
    z0 = 1 - z1 - z2
    total = 0.0
    for za, zb, x2sq in ((z1, z0, x02sq), (z0, z1, x21sq)):
        M2 = Q2 * za * (1 - za) + mf * mf
        total = total - za**2 * (2 * zb * (zb + z2) + z2**2) / x2sq * np.exp(-x2sq / x01sq / E_GAMMA) * k0(
            np.sqrt(M2) * np.sqrt(x01sq)) ** 2
    return 4 * Q2 * total


def l_qg_i2(t: Tripole, Q2, mf, G):
    z0, z1, z2 = t.z0, t.z1, t.z2
    b = [k0(np.sqrt(t.Qb2[s] + mf * mf) * np.sqrt(_X2(t, s))) for s in (0, 1)]
    x02sq, x21sq = t.x2sq
    return 4 * Q2 * (
        z1**2 * (2 * z0 * (z0 + z2) + z2**2) / 4 * G[("12", 0)] * b[0]
        + z0**2 * (2 * z1 * (z1 + z2) + z2**2) / 4 * G[("12", 1)] * b[1]
        - z0 * z1 * (z0 * (1 - z0) + z1 * (1 - z1)) * t.x20x21 / 4
        * (G[("12", 0)] * b[1] / x21sq + G[("12", 1)] * b[0] / x02sq))


def l_qg_i3(t: Tripole, Q2, mf, G1, G2):
    z0, z1, z2 = t.z0, t.z1, t.z2
    x02sq, x21sq = t.x2sq
    return 4 * Q2 * (
        z1**2 * (2 * z0 * (z0 + z2) + z2**2) * x02sq / 64 * G1[("12", 0)] * G2[("12", 0)]
        + z0**2 * (2 * z1 * (z1 + z2) + z2**2) * x21sq / 64 * G1[("12", 1)] * G2[("12", 1)]
        - z1 * z0 * (z1 * (1 - z1) + z0 * (1 - z0)) * t.x20x21 / 32 * G1[("12", 0)] * G2[("12", 1)]
        + mf * mf / 16 * z2**4 * ((z1 / (z0 + z2)) ** 2 * G1[("11", 0)] * G2[("11", 0)]
                                 + (z0 / (z1 + z2)) ** 2 * G1[("11", 1)] * G2[("11", 1)]
                                 - 2 * z0 / (z1 + z2) * z1 / (z0 + z2) * G1[("11", 0)] * G2[("11", 1)]))


def nested_rule(points=48):
    """y = t^3 map of the Gauss-Legendre rule on t in [0, 1] (custom_kernels/dis/i2_i3/extension.py:21-35)."""
    nodes, weights = np.polynomial.legendre.leggauss(points)
    t = (nodes + 1) / 2
    return t**3, weights / 2 * 3 * t**2


def nested_moments(t: Tripole, mf, points=48):
    ys, ws = nested_rule(points)
    moments = None
    for y, w in zip(ys, ws):
        G = t_moments_at(t, mf, np.full_like(t.z0, y))
        if moments is None:
            moments = {k: w * v for k, v in G.items()}
        else:
            for k in moments:
                moments[k] = moments[k] + w * G[k]
    return moments


def qg_rapidity(Q2, xbj, z2):
    return np.log(Q2 / xbj * z2 / Q0SQR)


def tripole_amplitude(dipole, x01, x02, x21, Y, finite_nc):
    S01 = 1 - dipole(x01, Y)
    S02 = 1 - dipole(x02, Y)
    S12 = 1 - dipole(x21, Y)
    if finite_nc:
        return 1 - NC / (2 * CF) * (S02 * S12 - S01 / NC**2)
    return 1 - S02 * S12


QG_DIMS = {"I1": 5, "I2": 6, "I3": 7, "I2n": 5, "I3n": 5}


def qg_integrand(x, kin: Kinematics, contribution: str, dipole, points=48):
    """integrand_qgunsub_massive (dis/observables.py:175-250) for 'I1', 'I2', 'I3';
    the nested forms 'I2n', 'I3n' integrate the auxiliary variables with the inner rule
    (dis/observables.py:253-331)."""
    Q2, xbj, mf = kin.Q2, kin.xbj, kin.mf
    z2min = Q0SQR / (Q2 / xbj)
    if z2min > 1:
        return np.zeros(x.shape[0])
    z1 = (1 - z2min) * x[:, 0]
    z2 = (1 - z1 - z2min) * x[:, 1] + z2min
    x01 = kin.maxr * x[:, 2]
    x02 = kin.maxr * x[:, 3]
    phi = 2 * math.pi * x[:, 4]
    x01sq = x01 * x01
    x02sq = x02 * x02
    x21sq = np.maximum(x01sq + x02sq - 2 * x01 * x02 * np.cos(phi), 0)
    x21 = np.sqrt(x21sq)
    jac = (1 - z2min) * (1 - z1 - z2min) * x01 * x02 * kin.maxr**2 * 2 * math.pi
    Y = qg_rapidity(Q2, xbj, z2)
    Ye = np.maximum(Y, 0)
    with np.errstate(all="ignore"):
        N012 = tripole_amplitude(dipole, x01, x02, x21, Ye, kin.finite_nc)
        r_alpha = x01 if kin.parent_coupling else np.minimum(x01, np.minimum(x02, x21))
        af = alpha_bar(r_alpha, kin)
        if contribution == "I1":
            N01 = dipole(x01, Ye)
            if kin.transverse:
                v = (N01 * t_qg_dipole_uvsub(Q2, mf, z1, z2, x01sq, x02sq, x21sq)
                     + N012 * t_qg_tripole_i1(Q2, mf, z1, z2, x01sq, x02sq, x21sq))
            else:
                v = (N01 * l_qg_dipole_uvsub(Q2, mf, z1, z2, x01sq, x02sq, x21sq)
                     + N012 * l_qg_tripole_i1(Q2, mf, z1, z2, x01sq, x02sq, x21sq))
        else:
            t = tripole(Q2, z1, z2, x01sq, x02sq, x21sq)
            if contribution in ("I2", "I3"):
                G1 = t_moments_at(t, mf, x[:, 5])
                G2 = t_moments_at(t, mf, x[:, 6]) if contribution == "I3" else None
            else:
                G1 = G2 = nested_moments(t, mf, points)
            if contribution in ("I2", "I2n"):
                v = t_qg_i2(t, mf, G1) if kin.transverse else l_qg_i2(t, Q2, mf, G1)
            else:
                v = t_qg_i3(t, mf, G1, G2) if kin.transverse else l_qg_i3(t, Q2, mf, G1, G2)
            v = N012 * v
        out = v * jac * af / z2
    return np.where((Y >= 0) & np.isfinite(out), out, 0.0)


# ----------------------------------------------------------------------------- integration


def gauss_legendre_tensor(f, dims, points):
    """Unit-cube tensor Gauss-Legendre value (numerics/integration.py:94-117 without the
    error estimate)."""
    nodes, weights = np.polynomial.legendre.leggauss(points)
    u = (nodes + 1) / 2
    w = weights / 2
    grids = np.meshgrid(*([u] * dims), indexing="ij")
    wgrids = np.meshgrid(*([w] * dims), indexing="ij")
    x = np.stack([g.reshape(-1) for g in grids], axis=1)
    wt = np.prod(np.stack([g.reshape(-1) for g in wgrids], axis=1), axis=1)
    return float(np.sum(wt * f(x)))


def vegas_map(edges, bin_index, frac):
    """x = left + width * frac per dimension and the inverse density prod(bins * width)."""
    bins = edges.shape[1] - 1
    d = np.arange(edges.shape[0])
    left = edges[d, bin_index]
    width = edges[d, bin_index + 1] - left
    return left + width * frac, np.prod(bins * width, axis=1)


def adapt_edges(edges, histogram, count):
    """_adapt_vegas_edges (numerics/integration.py:804-866), float64."""
    bins = histogram.shape[1]
    imp = histogram / np.maximum(count, 1)
    sm = imp.copy()
    sm[:, 1:-1] = (imp[:, :-2] + imp[:, 1:-1] + imp[:, 2:]) / 3
    sm[:, 0] = (imp[:, 0] + imp[:, 1]) / 2
    sm[:, -1] = (imp[:, -2] + imp[:, -1]) / 2
    sm = sm + np.finfo(np.float64).eps
    out = np.empty_like(edges)
    for d in range(edges.shape[0]):
        cum = np.concatenate(([0.0], np.cumsum(sm[d])))
        target = np.linspace(0, cum[-1], bins + 1)
        idx = np.clip(np.searchsorted(cum, target, side="right") - 1, 0, bins - 1)
        frac = (target - cum[idx]) / sm[d, idx]
        up = edges[d, idx] + frac * (edges[d, idx + 1] - edges[d, idx])
        up[0] = 0
        up[-1] = 1
        out[d] = up
    return out


def vegas_iteration(f, edges, bin_index, frac):
    """One Vegas iteration on given (bin, fraction) samples: the weighted sums, the
    histogram of |weight| and the bin counts (numerics/integration.py:240-489)."""
    x, inv = vegas_map(edges, bin_index, frac)
    w = f(x) * inv
    dims, bins = edges.shape[0], edges.shape[1] - 1
    hist = np.zeros((dims, bins))
    count = np.zeros((dims, bins))
    for d in range(dims):
        hist[d] = np.bincount(bin_index[:, d], weights=np.abs(w), minlength=bins)
        count[d] = np.bincount(bin_index[:, d], minlength=bins)
    return float(np.sum(w)), float(np.sum(w * w)), hist, count


def vegas(f, dims, sampler, *, samples, max_iterations, min_iterations=1, bins=32,
          warmup_samples=0, epsrel=0.2, epsabs=0.0):
    """Vegas driver of numerics/integration.py:120-589 on samples from `sampler(i, n)`,
    which returns (bin_index [n, dims] int, fraction [n, dims]) for iteration i.
    Returns (value, error, n_eval, converged, edges)."""
    edges = np.tile(np.linspace(0, 1, bins + 1), (dims, 1))
    estimates, variances = [], []
    n_eval = 0
    converged = False
    value = error = 0.0
    iterations = max_iterations + int(warmup_samples > 0)
    for it in range(iterations):
        warm = warmup_samples > 0 and it == 0
        n = warmup_samples if warm else samples
        bi, fr = sampler(it, n)
        total, total2, hist, count = vegas_iteration(f, edges, bi, fr)
        n_eval += n
        edges = adapt_edges(edges, hist, count)
        if warm:
            continue
        est = total / n
        var = max(max(total2 - total * total / n, 0.0) / (n - 1) / n, np.finfo(np.float64).tiny)
        estimates.append(est)
        variances.append(var)
        wts = 1 / np.array(variances)
        value = float(np.sum(wts * np.array(estimates)) / wts.sum())
        error = float(math.sqrt(1 / wts.sum()))
        converged = len(estimates) >= min_iterations and error <= max(epsabs, epsrel * abs(value))
        if converged:
            break
    return value, error, n_eval, converged, edges


def sobol_sampler(points, bins):
    """Map unit-cube points to Vegas (bin, fraction) pairs: bin = floor(u bins), the
    fraction the remainder (the same split as dis/fixed_sobol.py:101-112)."""
    scaled = points * bins
    bi = np.minimum(np.floor(scaled).astype(np.int64), bins - 1)
    return bi, scaled - bi


LO_FACTOR = 4 * ALPHA_EM * NC / (2 * math.pi) ** 2
DIP_FACTOR = 4 * NC * ALPHA_EM / (2 * math.pi) ** 2 * 2 * math.pi
QG_FACTOR = 4 * NC * ALPHA_EM / (2 * math.pi) ** 3 * 2 * math.pi


def structure_function_factor(Q2, transverse_area=1.0):
    """sigma -> F (dis/observables.py:535-561)."""
    return Q2 / (4 * math.pi**2 * ALPHA_EM) * transverse_area


def reduced_cross_section(F2, FL, Q2, xbj, sqrt_s):
    y = Q2 / (sqrt_s**2 * xbj)
    return F2 - y * y / (1 + (1 - y) ** 2) * FL


# ----------------------------------------------------------------------------- fixed-Sobol qg path


def map_importance_grid(points, edges):
    """Unit points through the importance grid: source, inverse density and bins
    (dis/fixed_sobol.py:100-112)."""
    bins = edges.shape[1] - 1
    scaled = points * bins
    bi = np.minimum(np.floor(scaled).astype(np.int64), bins - 1)
    frac = scaled - bi
    d = np.arange(edges.shape[0])
    left = edges[d, bi]
    width = edges[d, bi + 1] - left
    return left + width * frac, np.prod(bins * width, axis=1), bi


def paired_endpoint_inputs(source, maxr, fold_angle=False):
    """Split the gluon plane by the nearer dipole end (dis/fixed_sobol.py:115-158): the
    two 5D inputs and their weights."""
    parent = maxr * source[:, 2]
    radial = source[:, 3]
    af = 0.5 * source[:, 4] if fold_angle else source[:, 4]
    angle = 2 * np.pi * af
    c, s = np.cos(angle), np.sin(angle)
    tiny = np.finfo(np.float64).tiny
    with np.errstate(divide="ignore"):
        closer = np.where(c > 0, parent / (2 * np.maximum(c, tiny)), np.inf)
    first_limit = np.minimum(maxr, closer)
    first = source.copy()
    first[:, 3] = radial * first_limit / maxr
    first[:, 4] = af
    first_weight = first_limit / maxr
    disk = parent * c + np.sqrt(np.maximum(maxr**2 - parent**2 * s**2, 0))
    second_limit = np.maximum(np.minimum(disk, closer), 0)
    sr = radial * second_limit
    gx, gy = parent - sr * c, sr * s
    gr = np.sqrt(gx**2 + gy**2)
    second = source.copy()
    second[:, 3] = gr / maxr
    second[:, 4] = np.remainder(np.arctan2(gy, gx), 2 * np.pi) / (2 * np.pi)
    second_weight = sr * second_limit / (np.maximum(gr, tiny) * maxr)
    return first, first_weight, second, second_weight


def qg_triple(x, kin: Kinematics, dipole, points=48):
    """(I1, I2, I3) at x: the un-nested I1 and the nested I2, I3."""
    return (qg_integrand(x, kin, "I1", dipole), qg_integrand(x, kin, "I2n", dipole, points),
            qg_integrand(x, kin, "I3n", dipole, points))


def fixed_sobol(triple, training, replicates, maxr, bins=32, fold_angle=True, i1_weight=1.0):
    """learn_triple_importance_grid (dis/fixed_sobol.py:161-211) then the replicate
    estimates of integrate_triple_fixed_sobol (:214-270).  Returns (edges, estimates
    [replicates, 3])."""
    dims = training[0].shape[1]
    edges = np.tile(np.linspace(0, 1, bins + 1), (dims, 1))
    tiny = np.finfo(np.float64).tiny
    for pts in training:
        source, inv, bi = map_importance_grid(pts, edges)
        first, fw, second, sw = paired_endpoint_inputs(source, maxr, fold_angle)
        v1, v2 = triple(first), triple(second)
        weighted = [(a * fw + b * sw) * inv for a, b in zip(v1, v2)]
        score = sum(w * np.abs(v) / max(np.abs(v).mean(), tiny)
                    for w, v in zip((i1_weight, 1.0, 1.0), weighted))
        hist = np.zeros((dims, bins))
        count = np.zeros((dims, bins))
        for d in range(dims):
            hist[d] = np.bincount(bi[:, d], weights=score, minlength=bins)
            count[d] = np.bincount(bi[:, d], minlength=bins)
        edges = adapt_edges(edges, hist, count)
    estimates = []
    for pts in replicates:
        source, inv, _ = map_importance_grid(pts, edges)
        first, fw, second, sw = paired_endpoint_inputs(source, maxr, fold_angle)
        v1, v2 = triple(first), triple(second)
        estimates.append([float(np.mean((a * fw + b * sw) * inv)) for a, b in zip(v1, v2)])
    return edges, np.array(estimates)


def replicate_result(values):
    """Mean and standard error of replicate estimates (dis/fixed_sobol.py:258-268)."""
    values = np.asarray(values, dtype=np.float64)
    return float(values.mean()), float(values.std(ddof=1) / math.sqrt(values.size))
