// Device special functions and couplings of the NLO DIS integrands (sm_100a).
//
// Templated on the arithmetic type T (float: the mixed build; double: the all-FP64
// build).  The reference evaluates K0/K1 with torch.special (numerics/special.py:10-31)
// and Li2 with a 64-term power series (numerics/special.py:34-96); here:
//
// * K0 and K1 together (one log or one exp per pair): the ascending series for x <= 2
//   (Abramowitz & Stegun 9.6.10-9.6.11) and exp(-x) x^{-1/2} g_nu(2/x) above, with g_nu
//   a Chebyshev interpolant (FP64, Clenshaw) or a least-squares polynomial (FP32) fitted
//   by gen_special_tables.py against 50-digit values; relative error <= 1.3e-15 (FP64)
//   and <= 8e-7 (FP32) on (0, 500].
// * Li2 by the Bernoulli series in u = -ln(1-x) ('t Hooft & Veltman 1979) after the
//   inversion (x < -1) and reflection (x > 1/2) identities.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include "special_tables.cuh"

namespace nlo {
namespace dis {

constexpr double kPi = 3.14159265358979323846;
constexpr double kPi2Over6 = kPi * kPi / 6.0;
constexpr double kEulerGamma = 0.5772156649015329;
constexpr double kAlphaEM = 1.0 / 137.035999;
constexpr double kNc = 3.0;
constexpr double kCF = (kNc * kNc - 1.0) / (2.0 * kNc);
constexpr double kLambdaQCD = 0.241;
constexpr double kQ0sqr = 1.0;
constexpr double kZmin = 1e-6;

template <typename T>
struct DM;

template <>
struct DM<float> {
    static __device__ __forceinline__ float exp(float x) { return expf(x); }
    static __device__ __forceinline__ float log(float x) { return logf(x); }
    static __device__ __forceinline__ float log1p(float x) { return log1pf(x); }
    static __device__ __forceinline__ float expm1(float x) { return expm1f(x); }
    static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float rsqrt(float x) { return rsqrtf(x); }
    static __device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
    static __device__ __forceinline__ float pow(float x, float y) { return powf(x, y); }
    static __device__ __forceinline__ bool finite(float x) { return isfinite(x); }
};

template <>
struct DM<double> {
    static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
    static __device__ __forceinline__ double log(double x) { return ::log(x); }
    static __device__ __forceinline__ double log1p(double x) { return ::log1p(x); }
    static __device__ __forceinline__ double expm1(double x) { return ::expm1(x); }
    static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
    static __device__ __forceinline__ double rsqrt(double x) { return ::rsqrt(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double pow(double x, double y) { return ::pow(x, y); }
    static __device__ __forceinline__ bool finite(double x) { return isfinite(x); }
};

template <typename T, int N>
__device__ __forceinline__ T horner(const T (&c)[N], T t)
{
    T acc = c[N - 1];
#pragma unroll
    for (int i = N - 2; i >= 0; --i) acc = fma(acc, t, c[i]);
    return acc;
}

// Horner in v of the polynomial with coefficients c_k a^k b.  With a (a power of two) and
// b constants at the call site the scaled coefficients fold into the instructions, so a
// change of variable or an overall factor costs nothing at run time.
template <int N>
__device__ __forceinline__ float horner_scaled(const float (&c)[N], float a, float b, float v)
{
    float p[N];
    p[0] = b;
#pragma unroll
    for (int k = 1; k < N; ++k) p[k] = p[k - 1] * a;
    float acc = c[N - 1] * p[N - 1];
#pragma unroll
    for (int i = N - 2; i >= 0; --i) acc = fmaf(acc, v, c[i] * p[i]);
    return acc;
}

template <int N>
__device__ __forceinline__ double clenshaw(const double (&c)[N], double y)
{
    double b1 = 0.0, b2 = 0.0;
    const double y2 = 2.0 * y;
#pragma unroll
    for (int i = N - 1; i >= 1; --i) {
        const double b0 = fma(y2, b1, c[i] - b2);
        b2 = b1;
        b1 = b0;
    }
    return fma(y, b1, c[0] - b2);
}

template <typename T>
struct K01 {
    T k0, k1;
};

__device__ __forceinline__ K01<double> bessel_k01(double x)
{
    using namespace nlo_special;
    K01<double> out;
    if (x <= 2.0) {
        const double t = 0.25 * x * x;
        const double L = ::log(0.5 * x);
        out.k0 = fma(-L, horner(kI0Series, t), horner(kQ0Series, t));
        out.k1 = 1.0 / x + 0.5 * x * fma(L, horner(kI1Series, t), -0.5 * horner(kQ1Series, t));
    } else {
        const double y = 4.0 / x - 1.0;
        const double e = ::exp(-x) * ::rsqrt(x);
        out.k0 = e * clenshaw(kK0Cheb, y);
        out.k1 = e * clenshaw(kK1Cheb, y);
    }
    return out;
}

__device__ __forceinline__ float ex2_approx_f(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float lg2_approx_f(float x)
{
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rcp_approx_f(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// exp(-x) for x >= 0 from the hardware 2^x: x log2(e) is split into its rounded product
// and the exact rounding error (one FMA) plus the low part of log2(e), and 2^(-lo) is taken
// to first order; relative error about 3e-7 for every x up to the underflow.
__device__ __forceinline__ float exp_neg_f(float x)
{
    constexpr float kLog2eHi = 1.44269502162933349609375f;  // float(log2 e)
    constexpr float kLog2eLo = 1.925963033500011e-8f;        // log2 e - kLog2eHi
    const float hi = x * kLog2eHi;
    const float lo = fmaf(x, kLog2eHi, -hi) + x * kLog2eLo;
    return ex2_approx_f(-hi) * fmaf(-lo, 0.69314718055994531f, 1.0f);
}

// K0 and K1 from x and 1/x, FP32: the series in t = x^2/4 up to x = 2 (variable x^2, ln 2
// and the factors of K1 folded into the coefficients), e^-x/sqrt(x) times a polynomial in
// s = 2/x above (variable 1/x).  log(x/2) comes from the hardware log2 (absolute error
// near 1e-7), which near x = 2, where log(x/2) -> 0, bounds the relative error of K0 by
// about 3e-6; the FP32 build's integrals are held to 1e-4 of the FP64 ones.
__device__ __forceinline__ K01<float> bessel_k01_from_rcp(float x, float rx)
{
    using namespace nlo_special;
    constexpr float kLn2 = 0.69314718055994531f;
    K01<float> out;
    if (x <= 2.0f) {
        // K0 = -ln(x/2) I0(t) + Q0(t), K1 = 1/x + (x/2) (ln(x/2) I1(t) - Q1(t)/2), t = x^2/4,
        // with ln(x/2) = ln 2 (log2 x - 1)
        const float x2 = x * x;
        const float lg = lg2_approx_f(x) - 1.0f;
        out.k0 = fmaf(-lg, horner_scaled(kI0SeriesF, 0.25f, kLn2, x2), horner_scaled(kQ0SeriesF, 0.25f, 1.0f, x2));
        out.k1 = fmaf(x, fmaf(lg, horner_scaled(kI1SeriesF, 0.25f, 0.5f * kLn2, x2),
                              horner_scaled(kQ1SeriesF, 0.25f, -0.25f, x2)),
                      rx);
    } else {
        const float e = exp_neg_f(x) * rsqrtf(x);
        out.k0 = e * horner_scaled(kK0PolyF, 2.0f, 1.0f, rx);
        out.k1 = e * horner_scaled(kK1PolyF, 2.0f, 1.0f, rx);
    }
    return out;
}

__device__ __forceinline__ K01<float> bessel_k01(float x) { return bessel_k01_from_rcp(x, rcp_approx_f(x)); }

template <typename T>
__device__ __forceinline__ T bessel_k0(T x)
{
    return bessel_k01(x).k0;
}

template <typename T>
__device__ __forceinline__ T bessel_k1(T x)
{
    return bessel_k01(x).k1;
}

// Li2 on x <= 1 (numerics/special.py:34-96 domain).
template <typename T>
__device__ __forceinline__ T li2_core(T u)
{
    // sum_n B_n u^{n+1}/(n+1)! = u - u^2/4 + u^3 sum_k B_{2k}/(2k+1)! u^{2k-2}
    using namespace nlo_special;
    const T u2 = u * u;
    T series;
    if constexpr (sizeof(T) == 8)
        series = horner(kLi2Bernoulli, u2);
    else
        series = horner(kLi2BernoulliF, u2);
    return u - (T)0.25 * u2 + u * u2 * series;
}

template <typename T>
__device__ __forceinline__ T li2(T x)
{
    if (x == (T)1) return (T)kPi2Over6;
    if (x == (T)0) return (T)0;
    if (x < (T)-1) {
        // Li2(x) = -pi^2/6 - ln^2(-x)/2 - Li2(1/x)
        const T inv = (T)1 / x;
        const T lg = DM<T>::log(-x);
        return -(T)kPi2Over6 - (T)0.5 * lg * lg - li2_core(-DM<T>::log1p(-inv));
    }
    if (x > (T)0.5) {
        // Li2(x) = pi^2/6 - ln(x) ln(1-x) - Li2(1-x)
        const T y = (T)1 - x;
        return (T)kPi2Over6 - DM<T>::log(x) * DM<T>::log(y) - li2_core(-DM<T>::log1p(-y));
    }
    return li2_core(-DM<T>::log1p(-x));
}

// ---------------------------------------------------------------------------
// DIS couplings (coupling.py:49-97) and the alpha_s C_F / pi prefactor.
template <typename T>
struct Coupling {
    T b0;            // (11 Nc - 2 Nf)/(12 pi)
    T log_scale;     // log(4 C2 / Lambda^2)
    T max_alpha;     // freeze value
    T smooth_left;   // 2/0.2 * log(2.5)
    bool smooth;
};

template <typename T>
__device__ __forceinline__ T alpha_s(const Coupling<T>& c, T r)
{
    const T log_arg = c.log_scale - (T)2 * DM<T>::log(r);  // log(4 C2 / (r^2 Lambda^2))
    if (c.smooth) {
        const T right = log_arg * (T)5;  // / 0.2
        const T hi = right > c.smooth_left ? right : c.smooth_left;
        const T lo = right > c.smooth_left ? c.smooth_left : right;
        const T lae = hi + DM<T>::log1p(DM<T>::exp(lo - hi));
        return (T)1 / (c.b0 * (T)0.2 * lae);
    }
    const T a = (T)1 / (c.b0 * log_arg);
    return (a > c.max_alpha || log_arg < (T)0) ? c.max_alpha : a;
}

// GBW amplitude (dipole/amplitude.py:23-45).  The FP64 build keeps the reference's
// 1 - exp(-arg); FP32 uses -expm1(-arg), which avoids the cancellation at small arg.
template <typename T>
struct GBWParams {
    T qs0sqr, lambda, gamma, y0;
};

template <typename T>
__device__ __forceinline__ T gbw_amplitude(const GBWParams<T>& g, T r, T Y)
{
    const T Yeff = Y > g.y0 ? Y : g.y0;
    const T qs2 = g.qs0sqr * DM<T>::exp(g.lambda * Yeff);
    const T base = r * r * qs2;
    const T arg = (g.gamma == (T)1 ? base : DM<T>::pow(base, g.gamma)) * (T)0.25;
    if (arg < (T)1e-7) return arg;
    if constexpr (sizeof(T) == 8)
        return 1.0 - ::exp(-arg);
    else
        return -expm1f(-arg);
}

}  // namespace dis
}  // namespace nlo
