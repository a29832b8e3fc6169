"""Generate special_tables.cuh: coefficient tables of the device K0, K1 and Li2.

All coefficients are derived here from the mathematics, with mpmath at 50 digits
as the ground truth; nothing is taken from another library's tables.

* K0, K1 for x <= 2 use the ascending series (Abramowitz & Stegun 9.6.10-9.6.11)
      K0(x) = -ln(x/2) I0(x) + sum_k psi(k+1) t^k / (k!)^2,
      K1(x) = 1/x + ln(x/2) I1(x) - (x/4) sum_k (psi(k+1) + psi(k+2)) t^k / (k! (k+1)!),
  with t = x^2/4, I0 = sum t^k/(k!)^2 and I1 = (x/2) sum t^k/(k!(k+1)!).  The tables
  hold the exact series coefficients.
* K0, K1 for x > 2 use K_nu(x) = exp(-x) x^{-1/2} g_nu(2/x), where g_nu(s) is smooth on
  [0, 1] with g_nu(0) = sqrt(pi/2).  FP64: Chebyshev interpolant of g_nu in y = 2s - 1
  (Clenshaw recurrence on the device).  FP32: least-squares polynomial in s on Chebyshev
  nodes (Horner on the device).
* Li2 uses the Bernoulli-number series Li2(x) = sum_n B_n u^{n+1} / (n+1)!, u = -ln(1-x)
  ('t Hooft & Veltman, Nucl. Phys. B153 (1979) 365), after the standard reflection and
  inversion identities have brought x into [-1, 1/2].

* The double-log resummation factor of the BK kernel, J1(2 sqrt(-v))/sqrt(-v) for v < 0 and
  I1(2 sqrt(v))/sqrt(v) for v > 0, is one entire function G(v) = sum_k v^k / (k! (k+1)!).
  FP32 tables, t = 2 sqrt|v|, s = 4/t:
  - |v| <= 4: G = 1 + v q(v), q a least-squares polynomial (absolute error where |G| < 1,
    relative above);
  - v < -4: the modulus-phase form J1(t) = M1(t) cos(theta1(t)) (A&S 9.2.17), with
    M1 sqrt(pi t / 2) = m(s) and theta1 - (t - 3 pi/4) = d(s) least-squares polynomials in s;
  - v > 4: I1(t) = e^t / sqrt(2 pi t) h(s), h a least-squares polynomial in s (relative).

Run: python nlo_bk_optimized_b200/csrc/gen_special_tables.py  (writes special_tables.cuh
next to this file).
"""

from __future__ import annotations

from pathlib import Path

import mpmath as mp

mp.mp.dps = 50

SERIES_TERMS_F64 = 14
SERIES_TERMS_F32 = 8
CHEB_TERMS_F64 = 24
POLY_DEGREE_F32 = 9
BERNOULLI_TERMS_F64 = 20
BERNOULLI_TERMS_F32 = 9


def psi1(k: int):  # psi(k + 1) = -gamma + H_k
    return -mp.euler + sum(mp.mpf(1) / j for j in range(1, k + 1))


def series_tables(terms: int):
    i0 = [1 / mp.factorial(k) ** 2 for k in range(terms)]
    q0 = [psi1(k) / mp.factorial(k) ** 2 for k in range(terms)]
    i1 = [1 / (mp.factorial(k) * mp.factorial(k + 1)) for k in range(terms)]
    q1 = [(psi1(k) + psi1(k + 1)) / (mp.factorial(k) * mp.factorial(k + 1)) for k in range(terms)]
    return i0, q0, i1, q1


def g(nu: int, s):
    s = mp.mpf(s)
    if s == 0:
        return mp.sqrt(mp.pi / 2)
    x = 2 / s
    return mp.besselk(nu, x) * mp.exp(x) * mp.sqrt(x)


def chebyshev(nu: int, n: int):
    nodes = [mp.cos(mp.pi * (k + mp.mpf(1) / 2) / n) for k in range(n)]
    values = [g(nu, (t + 1) / 2) for t in nodes]
    coeffs = []
    for j in range(n):
        total = sum(values[k] * mp.cos(mp.pi * j * (k + mp.mpf(1) / 2) / n) for k in range(n))
        coeffs.append(2 * total / n)
    coeffs[0] /= 2
    return coeffs


def poly_fit(nu: int, degree: int):
    """Least-squares polynomial in s on 4*degree Chebyshev nodes of [0, 1], minimising
    the relative error."""
    m = 4 * (degree + 1)
    nodes = [(mp.cos(mp.pi * (k + mp.mpf(1) / 2) / m) + 1) / 2 for k in range(m)]
    A = mp.matrix(m, degree + 1)
    b = mp.matrix(m, 1)
    for i, s in enumerate(nodes):
        gv = g(nu, s)
        for j in range(degree + 1):
            A[i, j] = s**j / gv
        b[i] = 1
    coeffs = mp.lu_solve(A.T * A, A.T * b)
    return [coeffs[j] for j in range(degree + 1)]


DLA_T0 = 4  # t = 2 sqrt|v| where the polynomial hands over to the asymptotic forms
DLA_POLY_DEGREE = 8  # q(v)
DLA_J_DEGREE = 6     # m(s), d(s)
DLA_I_DEGREE = 8     # h(s)


def dla_g(v):
    v = mp.mpf(v)
    if v == 0:
        return mp.mpf(1)
    t = 2 * mp.sqrt(abs(v))
    return 2 * (mp.besselj(1, t) if v < 0 else mp.besseli(1, t)) / t


def least_squares(xs, targets, basis, weights, degree: int):
    A = mp.matrix(len(xs), degree + 1)
    b = mp.matrix(len(xs), 1)
    for i, (x, f, w) in enumerate(zip(xs, targets, weights)):
        for j in range(degree + 1):
            A[i, j] = basis(x, j) * w
        b[i] = f * w
    coeffs = mp.lu_solve(A.T * A, A.T * b)
    return [coeffs[j] for j in range(degree + 1)]


def cheb_nodes(a, b, m: int):
    return [a + (b - a) * (mp.cos(mp.pi * (k + mp.mpf(1) / 2) / m) + 1) / 2 for k in range(m)]


def dla_tables():
    v0 = mp.mpf(DLA_T0) ** 2 / 4
    vs = cheb_nodes(-v0, v0, 8 * (DLA_POLY_DEGREE + 1))
    gs = [dla_g(v) for v in vs]
    q = least_squares(vs, [g - 1 for g in gs], lambda v, j: v ** (j + 1), [1 / max(1, abs(g)) for g in gs],
                      DLA_POLY_DEGREE)
    ss = cheb_nodes(mp.mpf(0), mp.mpf(1), 8 * (DLA_I_DEGREE + 1))

    def modulus_phase(s):
        t = DLA_T0 / s
        j, y = mp.besselj(1, t), mp.bessely(1, t)
        d = mp.atan2(y, j) - (t - 3 * mp.pi / 4)
        return mp.sqrt(j * j + y * y) * mp.sqrt(mp.pi * t / 2), d - 2 * mp.pi * mp.nint(d / (2 * mp.pi))

    mdv = [modulus_phase(s) for s in ss]
    power = lambda s, j: s**j  # noqa: E731
    m = least_squares(ss, [x[0] for x in mdv], power, [1] * len(ss), DLA_J_DEGREE)
    d = least_squares(ss, [x[1] for x in mdv], power, [1] * len(ss), DLA_J_DEGREE)
    hv = [mp.besseli(1, DLA_T0 / s) * mp.sqrt(2 * mp.pi * DLA_T0 / s) * mp.exp(-DLA_T0 / s) for s in ss]
    h = least_squares(ss, hv, power, [1 / x for x in hv], DLA_I_DEGREE)
    return q, m, d, h


def bernoulli_tables(terms: int):
    # Li2 = u - u^2/4 + sum_{n>=1} B_{2n} u^{2n+1} / (2n+1)!
    return [mp.bernoulli(2 * n) / mp.factorial(2 * n + 1) for n in range(1, terms + 1)]


def fmt(values, suffix="") -> str:
    items = [mp.nstr(v, 20, min_fixed=-1, max_fixed=-1) + suffix for v in values]
    lines = []
    for i in range(0, len(items), 3):
        lines.append("    " + ", ".join(items[i : i + 3]) + ",")
    return "\n".join(lines)


def main() -> None:
    i0, q0, i1, q1 = series_tables(SERIES_TERMS_F64)
    out = [
        "// Generated by gen_special_tables.py; do not edit.  Derivation in that script.",
        "#pragma once",
        "",
        "namespace nlo_special {",
        "",
        f"constexpr int kSeriesTermsF64 = {SERIES_TERMS_F64};",
        f"constexpr int kSeriesTermsF32 = {SERIES_TERMS_F32};",
        f"constexpr int kChebTermsF64 = {CHEB_TERMS_F64};",
        f"constexpr int kPolyDegreeF32 = {POLY_DEGREE_F32};",
        f"constexpr int kBernoulliTermsF64 = {BERNOULLI_TERMS_F64};",
        f"constexpr int kBernoulliTermsF32 = {BERNOULLI_TERMS_F32};",
        "",
    ]
    for name, table in (("kI0Series", i0), ("kQ0Series", q0), ("kI1Series", i1), ("kQ1Series", q1)):
        out += [f"__device__ constexpr double {name}[{SERIES_TERMS_F64}] = {{", fmt(table), "};"]
    for name, table in (("kI0Series", i0), ("kQ0Series", q0), ("kI1Series", i1), ("kQ1Series", q1)):
        short = table[:SERIES_TERMS_F32]
        out += [f"__device__ constexpr float {name}F[{SERIES_TERMS_F32}] = {{", fmt(short, "f"), "};"]
    for nu in (0, 1):
        out += [f"__device__ constexpr double kK{nu}Cheb[{CHEB_TERMS_F64}] = {{",
                fmt(chebyshev(nu, CHEB_TERMS_F64)), "};"]
    for nu in (0, 1):
        out += [f"__device__ constexpr float kK{nu}PolyF[{POLY_DEGREE_F32 + 1}] = {{",
                fmt(poly_fit(nu, POLY_DEGREE_F32), "f"), "};"]
    out += [f"__device__ constexpr double kLi2Bernoulli[{BERNOULLI_TERMS_F64}] = {{",
            fmt(bernoulli_tables(BERNOULLI_TERMS_F64)), "};"]
    out += [f"__device__ constexpr float kLi2BernoulliF[{BERNOULLI_TERMS_F32}] = {{",
            fmt(bernoulli_tables(BERNOULLI_TERMS_F32), "f"), "};"]
    q, m, d, h = dla_tables()
    out += ["", f"constexpr float kDlaT0 = {DLA_T0}.0f;"]
    for name, table in (("kDlaPolyF", q), ("kDlaModF", m), ("kDlaPhaseF", d), ("kDlaExpF", h)):
        out += [f"__device__ constexpr float {name}[{len(table)}] = {{", fmt(table, "f"), "};"]
    out += ["", "}  // namespace nlo_special", ""]
    Path(__file__).with_name("special_tables.cuh").write_text("\n".join(out))


if __name__ == "__main__":
    main()
