// Shared device mathematics for the NLO BK kernels (sm_100a).
//
// Every kernel is templated on the arithmetic type T:
//   T = float  : the mixed build -- integrands in FP32 on the FMA/MUFU pipes,
//                FP32 partial sums of 32 samples folded into FP64 (K2+Kf), FP64
//                sums (K1);
//   T = double : the all-FP64 build used to check parity at 1e-10.
// The formulas are the reference's (torch_nlo_clean/src/nlo_torch: bk_kernels/k1.py,
// k2.py, kf.py, bk/derivatives.py, coupling.py) rewritten in algebraically identical
// forms that have no catastrophic cancellation, so that FP32 keeps ~1e-6 relative
// accuracy for every parent size r:
//   X^2          = (r - z)^2 + 4 r z sin^2(theta/2)
//   XY2^2-X2Y^2  = r [ r (z'^2 - z^2) - 2 z z' (z' cos th - z cos th') ]
//   log(a/b)/(a-b) = 2 h(t)/(a+b),  h(t) = atanh(t)/t,  t = (a-b)/(a+b)
//   alpha_Y - alpha_X from log1p/expm1 of the exact X^2 - Y^2
//   N_A - N_B    = S_A expm1(p_B - p_A) from log-spline values p
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "../../include/nlo_b200.h"

namespace nlo {

constexpr double kPi = 3.14159265358979323846;
constexpr double kMinLog = -40.0;  // numerics/interpolation.py:8

// ---------------------------------------------------------------------------
// Precision traits: fast MUFU-based functions for float, libm for double.
template <typename T>
struct M;

template <>
struct M<float> {
    static __device__ __forceinline__ float log_fast(float x) { return __logf(x); }
    static __device__ __forceinline__ float exp_fast(float x) { return __expf(x); }
    static __device__ __forceinline__ float log_acc(float x) { return logf(x); }
    static __device__ __forceinline__ float exp_acc(float x) { return expf(x); }
    // e^x - 1: (e^x - 1)/x as a degree-6 polynomial on [-1/2, 1/2] (least squares in
    // relative error at Chebyshev nodes, 3e-9; 1.3e-7 after FP32 Horner), the MUFU
    // exponential minus 1 outside, where no cancellation occurs.
    static __device__ __forceinline__ float expm1(float x)
    {
        float q = 0.00019823966831129978f;
        q = fmaf(q, x, 0.0013997217938334417f);
        q = fmaf(q, x, 0.008333698847676367f);
        q = fmaf(q, x, 0.04166532151841506f);
        q = fmaf(q, x, 0.16666662318239217f);
        q = fmaf(q, x, 0.5000000415133041f);
        q = fmaf(q, x, 1.0000000006631342f);
        return fabsf(x) < 0.5f ? x * q : __expf(x) - 1.0f;
    }
    // log(1 + v) = 2 atanh(s), s = v/(2 + v): atanh(s)/s as a degree-4 polynomial in s^2 on
    // [0, 1/9] (|v| <= 1/2; 4e-9, 2.1e-7 in FP32), the MUFU logarithm of 1 + v outside.
    static __device__ __forceinline__ float log1p(float v)
    {
        const float s = __fdividef(v, 2.0f + v);
        const float u = s * s;
        float p = 0.14080726880347302f;
        p = fmaf(p, u, 0.13982172352285377f);
        p = fmaf(p, u, 0.20012325666926623f);
        p = fmaf(p, u, 0.33333160203202167f);
        p = fmaf(p, u, 1.000000003861989f);
        return fabsf(v) <= 0.5f ? 2.0f * s * p : __logf(1.0f + v);
    }
    static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
    static __device__ __forceinline__ float sqrt(float x)
    {
        float y;
        asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
        return y;
    }
    static __device__ __forceinline__ float sin(float x) { return sinf(x); }
    static __device__ __forceinline__ float cos(float x) { return cosf(x); }
    static __device__ __forceinline__ float fmin(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float fmax(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float fabs(float a) { return fabsf(a); }
    static __device__ __forceinline__ bool finite(float a) { return isfinite(a); }
    // explicitly rounded map operations (the oracle replays them in float32)
    static __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
    static constexpr float tiny_square() { return 1e-38f; }
};

template <>
struct M<double> {
    static __device__ __forceinline__ double log_fast(double x) { return ::log(x); }
    static __device__ __forceinline__ double exp_fast(double x) { return ::exp(x); }
    static __device__ __forceinline__ double log_acc(double x) { return ::log(x); }
    static __device__ __forceinline__ double exp_acc(double x) { return ::exp(x); }
    static __device__ __forceinline__ double expm1(double x) { return ::expm1(x); }
    static __device__ __forceinline__ double log1p(double x) { return ::log1p(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double div(double a, double b) { return a / b; }
    static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
    static __device__ __forceinline__ double sin(double x) { return ::sin(x); }
    static __device__ __forceinline__ double cos(double x) { return ::cos(x); }
    static __device__ __forceinline__ double fmin(double a, double b) { return ::fmin(a, b); }
    static __device__ __forceinline__ double fmax(double a, double b) { return ::fmax(a, b); }
    static __device__ __forceinline__ double fabs(double a) { return ::fabs(a); }
    static __device__ __forceinline__ bool finite(double a) { return isfinite(a); }
    static __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
    static constexpr double tiny_square() { return 1e-40; }
};

// ---------------------------------------------------------------------------
// Physics constants, converted once per launch to the arithmetic type.
template <typename T>
struct Phys {
    T nc, nf, nf_over_nc;
    T b0c;        // b0 * 0.2 with b0 = (11 Nc - 2 Nf)/(12 pi)          coupling.py:92-96
    T left;       // 2/0.2 * log(2.5)                                     coupling.py:92
    T log_sc;     // log(4 C2 / Lambda^2)                                 coupling.py:94
    T log_4c2;    // log(4 C2), the heavy-flavour threshold coupling      coupling.py:25-45
    T fixed_as;   // fixed coupling value (if fixed), and the RESUM_RC_FIXED coupling
    T alpha_cap;  // > 0: cap
    T minr;
    T ksub, log_ksub;
    bool fixed;
    bool thresholds;  // NF > 3: bk_alpha_s with flavour thresholds (coupling.py:25-45)
    bool symmetrize;
    // BKConfig.Order / RC_LO / RESUM_RC / RC_NLO (nlo_bk_params)
    bool nlo;          // Order.has_nlo_kernels
    bool resum;        // Order.resum_dlog (k1.py:97-98: LO and NLO return the bare kernel)
    bool slog;         // Order.resum_slog
    int rc_lo;         // NLO_RC_LO_*
    int resum_rc;      // NLO_RESUM_RC_*
    bool nlo_parent;   // RC_NLO = PARENT_NLO
};

__host__ __device__ inline bool order_has_nlo(int order) { return order <= NLO_ORDER_NLO; }

template <typename T>
__host__ Phys<T> make_phys(const nlo_bk_params& p)
{
    Phys<T> q;
    q.nc = (T)p.nc;
    q.nf = (T)p.nf;
    q.nf_over_nc = (T)(p.nf / p.nc);
    q.b0c = (T)((11.0 * p.nc - 2.0 * p.nf) / (12.0 * kPi) * 0.2);
    q.left = (T)(2.0 / 0.2 * std::log(2.5));
    q.log_sc = (T)std::log(4.0 * p.c2 / (p.lambda_qcd * p.lambda_qcd));
    q.log_4c2 = (T)std::log(4.0 * p.c2);
    q.fixed_as = (T)p.fixed_alpha_s;
    q.alpha_cap = (T)p.alpha_cap;
    q.minr = (T)p.minr;
    q.ksub = (T)p.ksub;
    q.log_ksub = (T)std::log(p.ksub);
    q.fixed = p.fixed_coupling != 0;
    q.thresholds = !q.fixed && p.nf > 3.0;
    q.symmetrize = p.symmetrize != 0;
    q.nlo = order_has_nlo(p.order);
    q.resum = p.order != NLO_ORDER_NLO && p.order != NLO_ORDER_LO;
    q.slog = p.order == NLO_ORDER_NLO_RESUM_DLOG_SLOG || p.order == NLO_ORDER_LO_RESUM_DLOG_SLOG;
    q.rc_lo = p.rc_lo;
    q.resum_rc = p.resum_rc;
    q.nlo_parent = p.rc_nlo == NLO_RC_NLO_PARENT;
    return q;
}

// bk_alpha_s for NF > 3 (coupling.py:25-45): Nf = 3, 4, 5 below, between and above
// the scales 1.3 and 4.5 GeV of 4 C2 / d^2, with Lambda_Nf fixed per flavour number;
// 4 pi / (b0 log(4 C2 / (d^2 Lambda^2))), b0 = 11 - 2 Nf / 3, and 1 where the
// logarithm is negative or the coupling exceeds 1.
template <typename T>
__device__ __forceinline__ T alpha_thresholds(T log_d, const Phys<T>& ph)
{
    const T log_scale = ph.log_4c2 - (T)2 * log_d;  // log(4 C2 / d^2)
    T nf, log_lambda;
    if (log_scale < (T)0.5247285289349821) {         // log(1.3^2)
        nf = (T)3;
        log_lambda = (T)-1.9230602087529778;          // log(0.146159)
    } else if (log_scale < (T)3.0081547935525483) {  // log(4.5^2)
        nf = (T)4;
        log_lambda = (T)-2.0960263118360456;          // log(0.122944)
    } else {
        nf = (T)5;
        log_lambda = (T)-2.4030807944061756;          // log(0.0904389)
    }
    const T log_arg = log_scale - (T)2 * log_lambda;
    const T a = (T)(4.0 * kPi) * M<T>::rcp(((T)11 - (T)2 * nf / (T)3) * log_arg);
    return (log_arg < (T)0 || !(a <= (T)1)) ? (T)1 : a;
}

// logaddexp(left, right) with right = (log_sc - 2 log d)/0.2   (coupling.py:81-97)
template <typename T>
__device__ __forceinline__ T alpha_of_log(T log_d, const Phys<T>& ph)
{
    if (ph.fixed) return ph.fixed_as;
    if (ph.thresholds) return alpha_thresholds(log_d, ph);
    const T right = (ph.log_sc - (T)2 * log_d) * (T)5;
    const T m = M<T>::fmax(ph.left, right);
    const T lae = m + M<T>::log_fast((T)1 + M<T>::exp_fast(-M<T>::fabs(ph.left - right)));
    T a = M<T>::rcp(ph.b0c * lae);
    if (ph.alpha_cap > (T)0 && a > ph.alpha_cap) a = ph.alpha_cap;
    return a;
}

// ---------------------------------------------------------------------------
// Log-log spline in shared memory: knots x[n] (log r), coefficients (a,b,c,d) per interval.
// The r grid is logarithmically uniform, so the interval is found in O(1) from
// (lx - x0)/h.  FP64: a one-step fix-up against the stored knots gives the interval that
// searchsorted(x, lx, right=True) - 1 (clamped) would return (numerics/interpolation.py:70-76).
// FP32: the guess alone; it differs only within the FP32 rounding of lx from a knot, where
// the neighbouring piece is evaluated that far outside its interval -- the pieces join with
// continuous second derivatives, so the values agree to far below FP32 resolution.
template <typename T>
struct SplineView {
    const T* x;     // [n]
    const T* coef;  // [n-1][4]
    int n;
    T x0, inv_h;
};

__device__ __forceinline__ int floor_to_int(float v) { return __float2int_rd(v); }
__device__ __forceinline__ int floor_to_int(double v) { return __double2int_rd(v); }

template <typename T>
__device__ __forceinline__ int spline_interval(const SplineView<T>& s, T lx)
{
    int i = floor_to_int((lx - s.x0) * s.inv_h);
    i = i < 0 ? 0 : (i > s.n - 2 ? s.n - 2 : i);
    if constexpr (sizeof(T) == sizeof(double)) {
        if (i > 0 && lx < s.x[i]) --i;
        if (i < s.n - 2 && lx >= s.x[i + 1]) ++i;
    }
    return i;
}

template <typename T>
__device__ __forceinline__ T spline_poly(const SplineView<T>& s, T lx)
{
    const T lo = s.x[0], hi = s.x[s.n - 1];
    lx = lx < lo ? lo : (lx > hi ? hi : lx);
    const int i = spline_interval(s, lx);
    const T* c = s.coef + 4 * i;
    const T dx = lx - s.x[i];
    return c[0] + dx * (c[1] + dx * (c[2] + dx * c[3]));
}

// Amplitude at a distance with its log-S spline value (K2+Kf).
template <typename T>
struct NS {
    T p, N, S;
    int edge;  // -1 below r_min, 0 inside, +1 above r_max
};

// Edge rules of bk/derivatives.py:761-772 for the S row: S = 1 below r_min, 0 above r_max.
template <typename T>
__device__ __forceinline__ NS<T> eval_s_log(const SplineView<T>& s, T log_r)
{
    NS<T> v;
    if (log_r < s.x[0]) { v.p = (T)0; v.N = (T)0; v.S = (T)1; v.edge = -1; return v; }
    if (log_r > s.x[s.n - 1]) { v.p = (T)0; v.N = (T)1; v.S = (T)0; v.edge = 1; return v; }
    v.edge = 0;
    v.p = spline_poly(s, log_r);
    v.S = M<T>::exp_fast(v.p);
    v.N = -M<T>::expm1(v.p);
    return v;
}

// N_A - N_B
template <typename T>
__device__ __forceinline__ T ndiff_s(const NS<T>& A, const NS<T>& B)
{
    if (A.edge == 0 && B.edge == 0) return A.S * M<T>::expm1(B.p - A.p);
    if (A.N < (T)0.5 && B.N < (T)0.5) return A.N - B.N;
    return B.S - A.S;
}

// Per-evaluation variant without N: p and S only; N = -expm1(p) is formed in
// ndiff_ps only when one side is clamped to an edge value.
template <typename T>
struct PS {
    T p, S;
    int edge;
};

template <typename T>
__device__ __forceinline__ PS<T> eval_s_ps(const SplineView<T>& s, T log_r)
{
    PS<T> v;
    if (log_r < s.x[0]) { v.p = (T)0; v.S = (T)1; v.edge = -1; return v; }
    if (log_r > s.x[s.n - 1]) { v.p = (T)0; v.S = (T)0; v.edge = 1; return v; }
    v.edge = 0;
    v.p = spline_poly(s, log_r);
    v.S = M<T>::exp_fast(v.p);
    return v;
}

template <typename T>
__device__ __forceinline__ T n_of(const PS<T>& v)
{
    return v.edge < 0 ? (T)0 : (v.edge > 0 ? (T)1 : -M<T>::expm1(v.p));
}

template <typename T>
__device__ __forceinline__ T ndiff_ps(const PS<T>& A, const PS<T>& B)
{
    if (A.edge == 0 && B.edge == 0) return A.S * M<T>::expm1(B.p - A.p);
    const T NA = n_of(A), NB = n_of(B);
    if (NA < (T)0.5 && NB < (T)0.5) return NA - NB;
    return B.S - A.S;
}

// Spline value at lx minus the knot value a_i; Taylor form about knot i for lx in
// interval i or i-1 (no cancellation when lx is close to the knot).
template <typename T>
__device__ __forceinline__ T spline_delta_from_knot(const SplineView<T>& s, int i, T knot_value, T lx)
{
    const T lo = s.x[0], hi = s.x[s.n - 1];
    lx = lx < lo ? lo : (lx > hi ? hi : lx);
    const int j = spline_interval(s, lx);
    const T dx = lx - s.x[i];
    if (j == i) {
        const T* c = s.coef + 4 * i;
        return dx * (c[1] + dx * (c[2] + dx * c[3]));
    }
    if (j == i - 1) {
        const T* c = s.coef + 4 * (i - 1);
        const T h = s.x[i] - s.x[i - 1];
        const T b1 = c[1] + h * ((T)2 * c[2] + (T)3 * h * c[3]);
        const T c1 = c[2] + (T)3 * h * c[3];
        return dx * (b1 + dx * (c1 + dx * c[3]));
    }
    const T* c = s.coef + 4 * j;
    const T ddx = lx - s.x[j];
    const T pv = c[0] + ddx * (c[1] + ddx * (c[2] + ddx * c[3]));
    return pv - knot_value;
}

// Packed FP32x2 arithmetic of sm_100 (FFMA2/FADD2/FMUL2): two FP32 operations per
// instruction, component x and y.
using f2 = float2;
__device__ __forceinline__ f2 bc2(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 add2(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 sub2(f2 a, f2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ f2 mul2(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }

// M<float>::expm1 and M<float>::log1p for a pair.
__device__ __forceinline__ f2 expm1_2(f2 x)
{
    f2 q = fma2(bc2(0.00019823966831129978f), x, bc2(0.0013997217938334417f));
    q = fma2(q, x, bc2(0.008333698847676367f));
    q = fma2(q, x, bc2(0.04166532151841506f));
    q = fma2(q, x, bc2(0.16666662318239217f));
    q = fma2(q, x, bc2(0.5000000415133041f));
    q = fma2(q, x, bc2(1.0000000006631342f));
    const f2 p = mul2(x, q);
    return make_float2(fabsf(x.x) < 0.5f ? p.x : __expf(x.x) - 1.0f, fabsf(x.y) < 0.5f ? p.y : __expf(x.y) - 1.0f);
}
__device__ __forceinline__ f2 log1p_2(f2 v)
{
    const f2 sv = make_float2(__fdividef(v.x, 2.0f + v.x), __fdividef(v.y, 2.0f + v.y));
    const f2 u = mul2(sv, sv);
    f2 p = fma2(bc2(0.14080726880347302f), u, bc2(0.13982172352285377f));
    p = fma2(p, u, bc2(0.20012325666926623f));
    p = fma2(p, u, bc2(0.33333160203202167f));
    p = fma2(p, u, bc2(1.000000003861989f));
    const f2 r = mul2(add2(sv, sv), p);
    return make_float2(fabsf(v.x) <= 0.5f ? r.x : __logf(1.0f + v.x), fabsf(v.y) <= 0.5f ? r.y : __logf(1.0f + v.y));
}

// Compensated (Kahan) accumulation.
template <typename T>
struct Kahan {
    T sum, comp;
    __device__ __forceinline__ void reset() { sum = (T)0; comp = (T)0; }
    __device__ __forceinline__ void add(T v)
    {
        const T y = v - comp;
        const T t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
};

// Status word bits written by kernels (never a trap).
enum StatusBits : uint32_t {
    kStatusNonFinite = 1u << 0,
};

}  // namespace nlo
