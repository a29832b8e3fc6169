// K1: the LO-like part of the NLO BK right-hand side, by the fixed rule of
// custom_kernels/bk/k1/kernel.cu:2040-2092 (per r-grid interval 8 Gauss-Legendre
// nodes in log z times 24 nodes in v with theta = pi v^2, weight 2 z^2 * radial *
// pi v * angular), with the integrand Kernel_lo x dipole of bk_kernels/k1.py:20-155
// and bk/derivatives.py:434-468, for every Order, RC_LO and RESUM_RC of BKConfig
// (production: NLO_RESUM_DLOG_SLOG, BALITSKY_LO, RESUM_RC_SMALLEST).
//
// One CTA per active parent.  Threads own (interval, radial node) pairs and sweep
// the 24 angular nodes; per-thread sums are FP64, the block reduction is a fixed
// tree (deterministic).  In the mixed build the integrand runs in FP32 except on
// the two intervals adjacent to the parent knot (z -> x, where X -> 0 and the
// dipole N_Y - N_r cancels), which run in FP64.

#include <cooperative_groups.h>
#include <type_traits>
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "special_tables.cuh"

namespace cg = cooperative_groups;

namespace nlo {

namespace {

constexpr int kK1Threads = 256;
// Each parent's interval range is split over a cluster of CTAs; their partial
// sums are combined through distributed shared memory in rank order.
constexpr int kK1Split = 4;

// Log coordinates inside the kernel are measured from the parent knot: the spline
// knots are stored as x_j - log r (formed in FP64), and every distance enters as
// log(d/r).  In FP32 this keeps full relative precision of the amplitudes even where
// |log r| ~ 16, whose absolute FP32 spacing (2e-6) would otherwise become a 2e-6
// relative error of N.
template <typename T>
struct K1Parent {
    T r, r2;
    T lr_abs;      // log r (absolute), for the coupling
    T alpha_r;
    T Nr, Sr, pr;  // amplitude at the knot and its log value
    int knot;
};

// Amplitude at distance exp(lx) relative to the parent knot: N and D = N - N_r.
template <typename T>
__device__ __forceinline__ void k1_amplitude(const SplineView<T>& s, const K1Parent<T>& P, T lx, T& N, T& D)
{
    if (lx < s.x[0]) { N = (T)0; D = -P.Nr; return; }
    if (lx > s.x[s.n - 1]) { N = (T)1; D = P.Sr; return; }
    const T dp = spline_delta_from_knot(s, P.knot, P.pr, lx);
    const T pv = P.pr + dp;
    T nv = M<T>::exp_fast(pv);
    if (!M<T>::finite(nv)) nv = (T)0;
    if (nv >= (T)1) { N = (T)1; D = P.Sr; return; }
    N = nv;
    D = P.Nr * M<T>::expm1(dp);
}

// Per radial node (r-dependent but theta-independent) data.
template <typename T>
struct K1Z {
    T z, Ysq, inv_Ysq;
    T rho;        // z / r
    T dY;         // log(z / r)
    T NY, DY;
    T alpha_Y;
    T sigma, sigma_c;  // e^t/(e^c + e^t) and e^c/(e^c + e^t) at t = (log_sc - 2 log z)/0.2
};

// dlz = log z - log r (formed in FP64 by the caller), lz_abs = log z.
template <typename T>
__device__ __forceinline__ K1Z<T> k1_prepare_z(const SplineView<T>& s, const K1Parent<T>& P, const Phys<T>& ph,
                                              double dlz, double lz_abs)
{
    K1Z<T> Z;
    Z.dY = (T)dlz;
    Z.z = (T)::exp(lz_abs);
    Z.rho = (T)::exp(dlz);
    Z.Ysq = Z.z * Z.z;
    Z.inv_Ysq = M<T>::rcp(Z.Ysq);
    k1_amplitude(s, P, Z.dY, Z.NY, Z.DY);
    Z.alpha_Y = alpha_of_log((T)lz_abs, ph);
    const T right_Y = (ph.log_sc - (T)2 * (T)lz_abs) * (T)5;
    Z.sigma = M<T>::rcp((T)1 + M<T>::exp_fast(ph.left - right_Y));
    Z.sigma_c = M<T>::rcp((T)1 + M<T>::exp_fast(right_Y - ph.left));
    return Z;
}

// FP32 amplitude table of the production instantiation (mixed build, no kinematical
// constraint).  Rows in natural-log units over the uniform log r grid: row j + 1 =
// (a, b h, c h^2, d h^3) of interval j, so log N = a + t (b h + t (c h^2 + t d h^3)) with
// t = (log X - x_j)/h; row 0 = (-200, 0, 0, 0) below the grid (N = 0) and row n = (0, 0, 0, 0)
// above it (N = 1).  The position u = knot + log(X/r)/h picks the row with no search (the
// grid is uniform).  For the two intervals beside the parent knot, where X -> r and
// D = N_X - N_r must keep its relative precision, the per-parent rows rk (interval knot) and
// rkm1 (interval knot - 1 re-expanded about the knot) give log N - log N_r directly as a cubic
// without constant term in tau = log(X/r)/h, formed from log(X/r) itself.
struct K1Table {
    const float4* rows;  // [n + 1]
    float inv_h, knot;   // 1/h and the knot index (u of the parent)
    float top;           // n - 1
    float4 rk, rkm1;
};

// N and D = N - N_r at distance exp(lx) r (lx = log(X/r)): the row by selects, one exponential
// for N; D = N_r expm1(dp) near the knot (|dp| < 1/2, the polynomial of M<float>::expm1), else
// N - N_r; N >= 1 clamps to (1, S_r) as in k1_amplitude.
__device__ __forceinline__ void k1_amp_fast(const K1Table& t, const K1Parent<float>& P, float lx, float& N,
                                            float& D)
{
    const float u = fminf(fmaxf(fmaf(lx, t.inv_h, t.knot), -1.0f), t.top);
    // u + 2^23 + 1 rounded down is 2^23 + 1 + floor(u) (u >= -1): the row index sits in the low
    // mantissa bits, and subtracting the constant again gives floor(u) exactly
    const float shifted = __fadd_rd(u, 8388609.0f);
    const float jf = shifted - 8388609.0f;
    const float4 g = t.rows[__float_as_int(shifted) - 0x4B000000];
    const bool at_k = jf == t.knot, at_km1 = jf == t.knot - 1.0f;
    const bool near = at_k || at_km1;
    const float tau = near ? lx * t.inv_h : u - jf;
    const float4 c = at_k ? t.rk : (at_km1 ? t.rkm1 : make_float4(g.x - P.pr, g.y, g.z, g.w));
    const float dp = fmaf(tau, fmaf(tau, fmaf(tau, c.w, c.z), c.y), c.x);
    const float nv = __expf(P.pr + dp);
    float q = 0.00019823966831129978f;
    q = fmaf(q, dp, 0.0013997217938334417f);
    q = fmaf(q, dp, 0.008333698847676367f);
    q = fmaf(q, dp, 0.04166532151841506f);
    q = fmaf(q, dp, 0.16666662318239217f);
    q = fmaf(q, dp, 0.5000000415133041f);
    q = fmaf(q, dp, 1.0000000006631342f);
    const float d = fabsf(dp) < 0.5f ? P.Nr * (dp * q) : nv - P.Nr;
    const bool sat = nv >= 1.0f;
    N = sat ? 1.0f : nv;
    D = sat ? P.Sr : d;
}

// k1_prepare_z with the table's amplitude (the node is never beside the knot: those
// intervals are the FP64 panel's).
__device__ __forceinline__ K1Z<float> k1_prepare_z_fast(const K1Table& t, const K1Parent<float>& P,
                                                        const Phys<float>& ph, double dlz, double lz_abs)
{
    K1Z<float> Z;
    Z.dY = (float)dlz;
    Z.z = (float)::exp(lz_abs);
    Z.rho = (float)::exp(dlz);
    Z.Ysq = Z.z * Z.z;
    Z.inv_Ysq = M<float>::rcp(Z.Ysq);
    k1_amp_fast(t, P, Z.dY, Z.NY, Z.DY);
    Z.alpha_Y = alpha_of_log((float)lz_abs, ph);
    const float right_Y = (ph.log_sc - 2.0f * (float)lz_abs) * 5.0f;
    Z.sigma = M<float>::rcp(1.0f + M<float>::exp_fast(ph.left - right_Y));
    Z.sigma_c = M<float>::rcp(1.0f + M<float>::exp_fast(right_Y - ph.left));
    return Z;
}

// logaddexp(c, t + delta) - logaddexp(c, t) with the sigmoids of t precomputed.
template <typename T>
__device__ __forceinline__ T lae_shift(const K1Z<T>& Z, T delta)
{
    const T v = Z.sigma * M<T>::expm1(delta);
    if (v > (T)-0.5) return M<T>::log1p(v);
    return M<T>::log_acc(Z.sigma_c + Z.sigma * M<T>::exp_fast(delta));
}

// Kinematical constraint (bk/derivatives.py:469-487): the amplitude at distance d and the
// shifted rapidity y' from the stored history (_interpolate_history_N, :712-758).  Rows
// k and k+1 with y_k <= y' < y_{k+1} are each interpolated in r by the natural cubic
// spline through the 6 grid points starting at max(i-3, 0) (i the grid interval of d;
// d below the grid is moved to r_0 * 1.00001; a window past the grid gives 1), then
// linearly in y'; the result is clamped to [0, 1].  The spline's second derivatives
// are linear in the 6 values: kc_weights_kernel stores, per interval, the rows of that
// map for the two second derivatives the interval needs.
template <typename T>
__device__ __forceinline__ T kc_row_value(const double* row, const double* w, T h, T dx)
{
    T m0 = (T)0, m1 = (T)0, vj = (T)0, vj1 = (T)0;
    const int start = (int)w[0], j = (int)w[1];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const T v = (T)row[start + k];
        m0 += (T)w[2 + k] * v;
        m1 += (T)w[8 + k] * v;
        if (k == j) vj = v;
        if (k == j + 1) vj1 = v;
    }
    const T b = (vj1 - vj) / h - h * ((T)2 * m0 + m1) / (T)6;
    return vj + dx * (b + dx * (m0 / (T)2 + dx * (m1 - m0) / ((T)6 * h)));
}

// lx = log(d / r_parent) in the spline's coordinates (knots relative to the parent)
template <typename T>
__device__ __forceinline__ T kc_history_amplitude(const SplineView<T>& s, const K1History& H, const double* r_grid,
                                                  int n, T lx, int yind, T frac)
{
    if (lx >= s.x[n - 1]) return (T)1;  // rind = n-1: the window runs past the grid
    const bool below = lx < s.x[0];
    const int i = below ? 0 : spline_interval(s, lx);
    const double* w = H.weights + (size_t)i * kKcStride;
    if (w[0] < 0.0) return (T)1;
    const int node = (int)w[0] + (int)w[1];
    const double rj = r_grid[node];
    const T h = (T)(r_grid[node + 1] - rj);
    const T dx = below ? (T)(rj * 1.00001 - rj) : (T)rj * M<T>::expm1(lx - s.x[node]);
    const T lo = kc_row_value<T>(H.N + (size_t)yind * n, w, h, dx);
    const T hi = kc_row_value<T>(H.N + (size_t)(yind + 1) * n, w, h, dx);
    const T v = lo + frac * (hi - lo);
    return v < (T)0 ? (T)0 : (v > (T)1 ? (T)1 : v);
}

// The double-log resummation factor of Kernel_lo (k1.py:109-119): with
// x = 4 log(X/r) log(Y/r) and abar = alpha Nc / pi it is J1(2 sqrt(abar x))/sqrt(abar x) for
// x > 0 and I1(2 sqrt(abar |x|))/sqrt(abar |x|) for x < 0, i.e. G(v) at v = -abar x of the
// entire function G(v) = sum_k v^k / (k! (k+1)!) -- one function of one signed argument, so
// the two Bessel branches need no separate evaluation.  FP32: tables of
// gen_special_tables.py (mpmath fits) -- a polynomial for |v| <= 4, the modulus-phase form
// of J1 for v < -4 (one cosine after a Cody-Waite reduction of t = 2 sqrt|v| by a 2 pi split
// into an exact 8-bit part and the rest), e^t h(4/t) / sqrt(2 pi t) for v > 4 with e^t formed
// as two factors e^(t/2) so that only a value beyond the FP32 range overflows.  Error against
// G at the same FP32 t: 6e-7 of the envelope of G.
__device__ __forceinline__ float dla_factor(float v)
{
    using namespace nlo_special;
    const float av = fabsf(v);
    if (av <= 0.25f * kDlaT0 * kDlaT0) {
        float q = kDlaPolyF[8];
#pragma unroll
        for (int j = 7; j >= 0; --j) q = fmaf(q, v, kDlaPolyF[j]);
        return fmaf(v, q, 1.0f);
    }
    const float t = 2.0f * M<float>::sqrt(av);
    const float s = __fdividef(kDlaT0, t);
    const float srt = s * rsqrtf(t);  // 4 t^(-3/2)
    if (v < 0.0f) {
        float m = kDlaModF[6], d = kDlaPhaseF[6];
#pragma unroll
        for (int j = 5; j >= 0; --j) {
            m = fmaf(m, s, kDlaModF[j]);
            d = fmaf(d, s, kDlaPhaseF[j]);
        }
        // phase t - 3 pi/4 + d reduced to about [-pi, pi]: t - k (6.28125 + 2 pi - 6.28125)
        const float k = rintf(fmaf(t, 0.15915494309189535f, -0.375f));
        float rr = fmaf(-k, 6.28125f, t);  // exact: k 6.28125 has few bits and rr is representable
        rr = fmaf(-k, 1.9353071795864769e-3f, rr);
        rr = (rr - 2.3561944901923449f) + d;
        // 2 sqrt(2 / (pi t)) / t = sqrt(2 / pi) / 2 x 4 t^(-3/2)
        return (0.39894228040143268f * m) * srt * __cosf(rr);
    }
    float h = kDlaExpF[8];
#pragma unroll
    for (int j = 7; j >= 0; --j) h = fmaf(h, s, kDlaExpF[j]);
    const float half = __expf(0.5f * t);
    // 2 e^t / (t sqrt(2 pi t)) = 1 / (2 sqrt(2 pi)) x 4 t^(-3/2) x e^t
    return ((0.19947114020071634f * h) * srt * half) * half;
}

template <typename T>
__device__ __forceinline__ T dla_resum(T abar, T xarg);

template <>
__device__ __forceinline__ float dla_resum<float>(float abar, float xarg)
{
    return dla_factor(-abar * xarg);
}

// FP64: the Bessel functions themselves
template <>
__device__ __forceinline__ double dla_resum<double>(double abar, double xarg)
{
    const double as_x = ::sqrt(abar * ::fabs(xarg));
    if (as_x == 0.0) return 1.0;
    const double bes = xarg >= 0.0 ? ::j1(2.0 * as_x) : ::cyl_bessel_i1(2.0 * as_x);
    return bes / as_x;
}

// Kernel_lo x dipole at one (z, theta) node; sh2 = sin^2(theta/2).  The form of
// Kernel_lo follows RC_LO (k1.py:37-94); orders without resummation stop at the bare
// kernel (k1.py:97-98); the resummation coupling follows RESUM_RC (k1.py:100-107).
// F32_DLOG (the mixed build's FP64 panel nodes): the double-log factor from the FP32 G(v); the
// panel runs in FP64 for the cancellation of N_Y - N_r as z -> x, which that factor has no
// part in.
template <typename T, bool KC, bool F32_DLOG = false>
__device__ __forceinline__ T k1_point(const SplineView<T>& s, const K1Parent<T>& P, const K1Z<T>& Z,
                                      const Phys<T>& ph, T sh2, const K1History& H, const double* r_grid)
{
    const T r = P.r, z = Z.z;
    const T Xsq = (r - z) * (r - z) + (T)4 * r * z * sh2;
    if (!(Xsq >= M<T>::tiny_square())) return (T)0;
    // log(X/r) from (X/r)^2 = (1 - z/r)^2 + 4 (z/r) sin^2(theta/2)
    const T xr2 = ((T)1 - Z.rho) * ((T)1 - Z.rho) + (T)4 * Z.rho * sh2;
    const T dX = (T)0.5 * M<T>::log_fast(xr2);
    const T alpha_X = alpha_of_log(P.lr_abs + dX, ph);
    // X^2 - Y^2 = r (r - 2 z cos theta), cos theta = 1 - 2 sin^2(theta/2)
    const T XmY = r * (r - (T)2 * z * ((T)1 - (T)2 * sh2));
    // alpha_Y - alpha_X: the smooth coupling's difference without cancellation, else direct
    T dalpha;
    if (ph.fixed) {
        dalpha = (T)0;
    } else if (ph.alpha_cap > (T)0 || ph.thresholds) {
        dalpha = Z.alpha_Y - alpha_X;
    } else {
        // alpha_Y - alpha_X = alpha_X alpha_Y b0 c (lae_X - lae_Y)
        const T delta = -(T)5 * M<T>::log1p(XmY * Z.inv_Ysq);
        dalpha = alpha_X * Z.alpha_Y * ph.b0c * lae_shift(Z, delta);
    }
    const T inv_XY = M<T>::rcp(Xsq * Z.Ysq);
    const T pref = ph.nc * (T)(1.0 / (2.0 * kPi * kPi));
    // alpha at min(X, Y, r): reuse alpha_X, alpha_Y or alpha_r
    const T alpha_min = (dX <= Z.dY && dX <= (T)0) ? alpha_X : (Z.dY <= (T)0 ? Z.alpha_Y : P.alpha_r);
    T lo, alpha_sc;  // Kernel_lo and the coupling at its scale (alphas_scale)
    if (ph.rc_lo == NLO_RC_LO_PARENT) {
        alpha_sc = P.alpha_r;
        lo = pref * alpha_sc * P.r2 * inv_XY;
    } else if (ph.rc_lo == NLO_RC_LO_SMALLEST) {
        alpha_sc = alpha_min;
        lo = pref * alpha_sc * P.r2 * inv_XY;
    } else if (ph.rc_lo == NLO_RC_LO_FAC) {
        // 1/(2 pi) / (1/abar_r + (X^2-Y^2)/r^2 (abar_X - abar_Y)/(abar_X abar_Y)) r^2/(X^2 Y^2)
        //   = pref r^2/(X^2 Y^2) / (1/alpha_r - (X^2-Y^2)/r^2 (alpha_Y - alpha_X)/(alpha_X alpha_Y))
        alpha_sc = P.alpha_r;
        const T den = M<T>::rcp(P.alpha_r) - XmY * M<T>::rcp(P.r2) * M<T>::div(dalpha, alpha_X * Z.alpha_Y);
        lo = pref * P.r2 * inv_XY * M<T>::rcp(den);
    } else if (ph.rc_lo == NLO_RC_LO_BEUF) {
        // r_eff^2 = r^2 (Y^2/X^2)^((X^2-Y^2)/r^2): log r_eff = log r - (X^2-Y^2)/(2 r^2) log(X^2/Y^2)
        const T log_reff = P.lr_abs - (T)0.5 * XmY * M<T>::rcp(P.r2) * M<T>::log1p(XmY * Z.inv_Ysq);
        alpha_sc = alpha_of_log(log_reff, ph);
        lo = pref * alpha_sc * P.r2 * inv_XY;
    } else {
        // Balitsky: r^2/(X^2Y^2) + (aY/aX - 1)/Y^2 + (aX/aY - 1)/X^2
        alpha_sc = P.alpha_r;
        const T bracket =
            (P.r2 + dalpha * M<T>::div(Z.alpha_Y * XmY + Z.Ysq * dalpha, alpha_X * Z.alpha_Y)) * inv_XY;
        lo = pref * P.alpha_r * bracket;
    }
    if (!M<T>::finite(lo)) lo = (T)0;
    T dipole;
    // kinematical constraint: where min(X, Y) > r the daughters are taken at the shifted
    // rapidity y - log(min(X^2, Y^2)/r^2) from the history (zero when it is negative);
    // elsewhere the shift vanishes and the current amplitude is used
    const T dmin = M<T>::fmin(dX, Z.dY);
    if (KC && dmin > (T)0) {
        const double rapidity = H.y[H.rows - 1];
        const double shifted = rapidity - (double)((T)2 * dmin);
        if (shifted < 0.0) return (T)0;
        int lo = 0, hi = H.rows;  // yind = searchsorted(y, shifted, right) - 1
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (H.y[mid] <= shifted) lo = mid + 1; else hi = mid;
        }
        const int yind = lo - 1 < 0 ? 0 : lo - 1;
        if (yind >= H.rows - 1) {
            T NX, DX;  // at the current rapidity: the current amplitude
            k1_amplitude(s, P, dX, NX, DX);
            const T base = Z.NY <= NX ? Z.NY + DX : NX + Z.DY;
            dipole = P.Sr * base - DX * Z.DY;
        } else {
            const T frac = (T)((shifted - H.y[yind]) / (H.y[yind + 1] - H.y[yind]));
            const T NXh = kc_history_amplitude<T>(s, H, r_grid, s.n, dX, yind, frac);
            const T NYh = kc_history_amplitude<T>(s, H, r_grid, s.n, Z.dY, yind, frac);
            // (1 - N_r) - (1 - N_X')(1 - N_Y') without forming the 1 - N
            dipole = NXh + NYh - P.Nr - NXh * NYh;
        }
    } else {
        // dipole N_X + N_Y - N_r - N_X N_Y = S_r (N_Y + D_X) - D_X D_Y  (or with X and Y exchanged)
        T NX, DX;
        k1_amplitude(s, P, dX, NX, DX);
        const T base = Z.NY <= NX ? Z.NY + DX : NX + Z.DY;
        dipole = P.Sr * base - DX * Z.DY;
    }
    if (!ph.resum) {
        const T bare = lo * dipole;
        return M<T>::finite(bare) ? bare : (T)0;
    }
    // double-log resummation (k1.py:109-119) with the RESUM_RC coupling
    const T alpha_res = ph.resum_rc == NLO_RESUM_RC_PARENT
                            ? P.alpha_r
                            : (ph.resum_rc == NLO_RESUM_RC_FIXED ? ph.fixed_as : alpha_min);
    const T xarg = (T)4 * dX * Z.dY;
    const T abar = alpha_res * ph.nc * (T)(1.0 / kPi);
    T dlog = F32_DLOG ? (T)dla_factor((float)(-abar * xarg)) : dla_resum<T>(abar, xarg);
    if (!(r > (T)1.01 * ph.minr)) dlog = (T)1;
    if (!M<T>::finite(dlog)) return (T)0;
    // single-log resummation (k1.py:121-132): exp(-abar A1 |log(ksub (r/minxy)^2)|) and its
    // first-order expansion, subtracted with the kernel at one power of the coupling
    T slog = (T)1, slog_exp = (T)0;
    if (ph.slog) {
        const T dminxy = M<T>::fmin(dX, Z.dY);
        slog_exp = -abar * (T)(11.0 / 12.0) * M<T>::fabs(ph.log_ksub - (T)2 * dminxy);
        slog = M<T>::exp_fast(slog_exp);
    }
    const T lo_single = pref * alpha_sc * P.r2 * inv_XY;
    const T k1fin = lo * alpha_sc * ph.nc * (T)(1.0 / (4.0 * kPi)) *
                    ((T)(67.0 / 9.0 - kPi * kPi / 3.0) - (T)(10.0 / 9.0) * ph.nf_over_nc);
    const T result = (dlog * slog * lo - lo_single * slog_exp + k1fin) * dipole;
    return M<T>::finite(result) ? result : (T)0;
}

// k1_point for two angles of one radial node (x: angle j, y: angle j + 1) in the mixed
// build without the kinematical constraint: the same arithmetic on the packed FP32x2
// instructions, with the per-angle transcendental and table operations per component.
__device__ __forceinline__ f2 k1_pair_point(const K1Table& s, const K1Parent<float>& P,
                                            const K1Z<float>& Z, const Phys<float>& ph, f2 sh2)
{
    const float r = P.r, z = Z.z;
    const f2 Xsq = fma2(bc2((float)4 * r * z), sh2, bc2((r - z) * (r - z)));
    const bool ok_x = Xsq.x >= M<float>::tiny_square(), ok_y = Xsq.y >= M<float>::tiny_square();
    if (!ok_x && !ok_y) return bc2(0.0f);
    const f2 xr2 = fma2(bc2(4.0f * Z.rho), sh2, bc2((1.0f - Z.rho) * (1.0f - Z.rho)));
    const f2 dX = mul2(bc2(0.5f), make_float2(__logf(xr2.x), __logf(xr2.y)));
    // X^2 - Y^2 = r (r - 2 z cos theta), cos theta = 1 - 2 sin^2(theta/2)
    const f2 XmY = mul2(bc2(r), fma2(bc2(-2.0f * z), fma2(bc2(-2.0f), sh2, bc2(1.0f)), bc2(r)));
    const f2 aY = bc2(Z.alpha_Y);
    // alpha_X, dalpha = alpha_Y - alpha_X and ratio = dalpha / (alpha_X alpha_Y)
    f2 alpha_X, dalpha, ratio;
    if (ph.fixed) {
        alpha_X = bc2(ph.fixed_as);
        dalpha = ratio = bc2(0.0f);
    } else if (ph.alpha_cap > 0.0f || ph.thresholds) {
        alpha_X = make_float2(alpha_of_log(P.lr_abs + dX.x, ph), alpha_of_log(P.lr_abs + dX.y, ph));
        dalpha = sub2(aY, alpha_X);
        ratio = make_float2(__fdividef(dalpha.x, alpha_X.x * Z.alpha_Y), __fdividef(dalpha.y, alpha_X.y * Z.alpha_Y));
    } else {
        // smooth coupling, 1/alpha = b0 c lae: 1/alpha_X - 1/alpha_Y = b0 c (lae_X - lae_Y) = ratio,
        // with lae_X - lae_Y from log1p/expm1 of the exact X^2 - Y^2 (no cancellation); so
        // alpha_X = 1/(1/alpha_Y + ratio) and dalpha = alpha_X alpha_Y ratio
        // the shift's exponent delta = -5 log(X^2/Y^2) enters only through e^delta - 1 =
        // (1 + eps)^-5 - 1, eps = (X^2 - Y^2)/Y^2; since (1 + eps)^5 - 1 = eps P(eps),
        // P = 5 + 10 eps + 10 eps^2 + 5 eps^3 + eps^4, it is -eps P(eps)/(1 + eps)^5 without
        // cancellation near X = Y, and 1/(1 + eps)^5 - 1 farther away
        const f2 eps = mul2(XmY, bc2(Z.inv_Ysq));
        const f2 op = add2(bc2(1.0f), eps);
        const f2 op2 = mul2(op, op);
        const f2 op5 = mul2(mul2(op2, op2), op);
        const f2 r5 = make_float2(__fdividef(1.0f, op5.x), __fdividef(1.0f, op5.y));
        f2 P = fma2(eps, bc2(1.0f), bc2(5.0f));
        P = fma2(P, eps, bc2(10.0f));
        P = fma2(P, eps, bc2(10.0f));
        P = fma2(P, eps, bc2(5.0f));
        const f2 near = mul2(mul2(eps, P), make_float2(-r5.x, -r5.y));
        const f2 em1 = make_float2(fabsf(eps.x) < 0.5f ? near.x : r5.x - 1.0f, fabsf(eps.y) < 0.5f ? near.y : r5.y - 1.0f);
        const f2 v = mul2(bc2(Z.sigma), em1);
        f2 shift = log1p_2(v);
        if (v.x <= -0.5f) shift.x = logf(Z.sigma_c + Z.sigma * r5.x);
        if (v.y <= -0.5f) shift.y = logf(Z.sigma_c + Z.sigma * r5.y);
        ratio = mul2(bc2(ph.b0c), shift);
        const f2 inv_aX = add2(bc2(__fdividef(1.0f, Z.alpha_Y)), ratio);
        alpha_X = make_float2(__fdividef(1.0f, inv_aX.x), __fdividef(1.0f, inv_aX.y));
        dalpha = mul2(mul2(alpha_X, aY), ratio);
    }
    const f2 inv_XY = make_float2(__fdividef(1.0f, Xsq.x * Z.Ysq), __fdividef(1.0f, Xsq.y * Z.Ysq));
    const float pref = ph.nc * (float)(1.0 / (2.0 * kPi * kPi));
    // alpha at min(X, Y, r): reuse alpha_X, alpha_Y or alpha_r
    const f2 alpha_min = make_float2((dX.x <= Z.dY && dX.x <= 0.0f) ? alpha_X.x : (Z.dY <= 0.0f ? Z.alpha_Y : P.alpha_r),
                                     (dX.y <= Z.dY && dX.y <= 0.0f) ? alpha_X.y : (Z.dY <= 0.0f ? Z.alpha_Y : P.alpha_r));
    const f2 r2iXY = mul2(bc2(P.r2), inv_XY);
    f2 lo, alpha_sc;
    if (ph.rc_lo == NLO_RC_LO_PARENT) {
        alpha_sc = bc2(P.alpha_r);
        lo = mul2(bc2(pref * P.alpha_r), r2iXY);
    } else if (ph.rc_lo == NLO_RC_LO_SMALLEST) {
        alpha_sc = alpha_min;
        lo = mul2(mul2(bc2(pref), alpha_min), r2iXY);
    } else if (ph.rc_lo == NLO_RC_LO_FAC) {
        alpha_sc = bc2(P.alpha_r);
        const f2 den = sub2(bc2(__fdividef(1.0f, P.alpha_r)), mul2(mul2(XmY, bc2(__fdividef(1.0f, P.r2))), ratio));
        lo = mul2(mul2(bc2(pref), r2iXY), make_float2(__fdividef(1.0f, den.x), __fdividef(1.0f, den.y)));
    } else if (ph.rc_lo == NLO_RC_LO_BEUF) {
        const f2 log_reff = fma2(mul2(bc2(-0.5f * __fdividef(1.0f, P.r2)), XmY), log1p_2(mul2(XmY, bc2(Z.inv_Ysq))),
                                 bc2(P.lr_abs));
        alpha_sc = make_float2(alpha_of_log(log_reff.x, ph), alpha_of_log(log_reff.y, ph));
        lo = mul2(mul2(bc2(pref), alpha_sc), r2iXY);
    } else {
        // Balitsky: r^2/(X^2Y^2) + (aY/aX - 1)/Y^2 + (aX/aY - 1)/X^2
        alpha_sc = bc2(P.alpha_r);
        // = (r^2 + dalpha (alpha_Y (X^2 - Y^2) + Y^2 dalpha) / (alpha_X alpha_Y)) / (X^2 Y^2)
        const f2 num = fma2(aY, XmY, mul2(bc2(Z.Ysq), dalpha));
        const f2 bracket = mul2(fma2(ratio, num, bc2(P.r2)), inv_XY);
        lo = mul2(bc2(pref * P.alpha_r), bracket);
    }
    lo = make_float2(isfinite(lo.x) ? lo.x : 0.0f, isfinite(lo.y) ? lo.y : 0.0f);
    // dipole N_X + N_Y - N_r - N_X N_Y = S_r (N_Y + D_X) - D_X D_Y  (or with X and Y exchanged)
    float NXx, DXx, NXy, DXy;
    k1_amp_fast(s, P, dX.x, NXx, DXx);
    k1_amp_fast(s, P, dX.y, NXy, DXy);
    const f2 DX = make_float2(DXx, DXy);
    const f2 base = make_float2(Z.NY <= NXx ? Z.NY + DXx : NXx + Z.DY, Z.NY <= NXy ? Z.NY + DXy : NXy + Z.DY);
    const f2 dipole = fma2(bc2(P.Sr), base, mul2(bc2(-Z.DY), DX));
    f2 result;
    if (!ph.resum) {
        result = mul2(lo, dipole);
    } else {
        // double-log resummation (k1.py:109-119) with the RESUM_RC coupling
        const f2 alpha_res = ph.resum_rc == NLO_RESUM_RC_PARENT
                                 ? bc2(P.alpha_r)
                                 : (ph.resum_rc == NLO_RESUM_RC_FIXED ? bc2(ph.fixed_as) : alpha_min);
        const f2 xarg = mul2(bc2(4.0f * Z.dY), dX);
        const f2 abar = mul2(alpha_res, bc2(ph.nc * (float)(1.0 / kPi)));
        const f2 v = mul2(abar, make_float2(-xarg.x, -xarg.y));
        f2 dlog = make_float2(dla_factor(v.x), dla_factor(v.y));
        if (!(r > 1.01f * ph.minr)) dlog = bc2(1.0f);
        // single-log resummation (k1.py:121-132)
        f2 slog = bc2(1.0f), slog_exp = bc2(0.0f);
        if (ph.slog) {
            const f2 dminxy = make_float2(fminf(dX.x, Z.dY), fminf(dX.y, Z.dY));
            const f2 arg = fma2(bc2(-2.0f), dminxy, bc2(ph.log_ksub));
            slog_exp = mul2(mul2(abar, bc2(-11.0f / 12.0f)), make_float2(fabsf(arg.x), fabsf(arg.y)));
            slog = make_float2(__expf(slog_exp.x), __expf(slog_exp.y));
        }
        const f2 lo_single = mul2(mul2(bc2(pref), alpha_sc), r2iXY);
        const float fin = ph.nc * (float)(1.0 / (4.0 * kPi)) *
                          ((float)(67.0 / 9.0 - kPi * kPi / 3.0) - (float)(10.0 / 9.0) * ph.nf_over_nc);
        const f2 k1fin = mul2(mul2(lo, alpha_sc), bc2(fin));
        const f2 core = add2(sub2(mul2(mul2(dlog, slog), lo), mul2(lo_single, slog_exp)), k1fin);
        result = mul2(core, dipole);
        if (!isfinite(dlog.x)) result.x = 0.0f;
        if (!isfinite(dlog.y)) result.y = 0.0f;
    }
    return make_float2(ok_x && isfinite(result.x) ? result.x : 0.0f, ok_y && isfinite(result.y) ? result.y : 0.0f);
}

template <typename T>
__device__ __forceinline__ K1Parent<T> k1_parent(const SplineView<T>& s, const Phys<T>& ph, double r, int knot)
{
    K1Parent<T> P;
    P.r = (T)r;
    P.lr_abs = (T)::log(r);
    P.r2 = P.r * P.r;
    P.alpha_r = alpha_of_log(P.lr_abs, ph);
    P.knot = knot;
    P.pr = s.coef[4 * (knot < s.n - 1 ? knot : s.n - 2)];
    if (knot == s.n - 1) {
        const T* c = s.coef + 4 * (s.n - 2);
        const T h = s.x[s.n - 1] - s.x[s.n - 2];
        P.pr = c[0] + h * (c[1] + h * (c[2] + h * c[3]));
    }
    const T e = M<T>::exp_fast(P.pr);
    P.Nr = e < (T)1 ? e : (T)1;
    P.Sr = P.pr < (T)0 ? -M<T>::expm1(P.pr) : (T)0;
    return P;
}

struct K1Consts {
    K1Rule rule;
    double sh2[24];  // sin^2(theta_j / 2), theta_j = pi v_j^2
    double aw[24];   // w_j pi v_j
};

// TF: arithmetic of the regular intervals (float in the mixed build); KC: the
// kinematical constraint (a separate instantiation keeps the history code out of the
// production kernel's registers).  Without the constraint four CTAs share an SM: 64
// registers a thread and about 51 KB of shared memory a CTA (the FP64 coefficients
// stay in global memory).  The dependent integrand chain is latency-bound, and the
// extra warps gain more than the few values spilled to the stack cost.
template <typename TF, bool KC>
__global__ void __cluster_dims__(1, kK1Split, 1) __launch_bounds__(kK1Threads, KC ? 1 : 4)
    k1_kernel(Phys<TF> phf, Phys<double> phd, K1Consts consts, K1History history,
                                                        const double* __restrict__ r_grid, int n,
                                                        const double* __restrict__ spline,
                                                        const int32_t* __restrict__ active,
                                                        const int32_t* __restrict__ count, double* __restrict__ out)
{
    // set blockIdx.z: its spline table, active list, count and output row
    spline += (size_t)blockIdx.z * spline_doubles(n);
    active += (size_t)blockIdx.z * n;
    count += blockIdx.z;
    out += (size_t)blockIdx.z * n;
    const int slot = blockIdx.x;
    if (slot >= *count) return;
    const int knot = active[slot];
    // this CTA's share of the radial nodes (contiguous interval ranges)
    const int nodes = (n - 1) * 8;
    const int split = blockIdx.y;
    const int per_split = ((n - 1 + kK1Split - 1) / kK1Split) * 8;
    const int k_begin = split * per_split;
    const int k_end = min(nodes, k_begin + per_split);
    const int k_count = max(0, k_end - k_begin);

    extern __shared__ __align__(16) unsigned char k1_smem[];
    unsigned char* cursor = k1_smem;
    auto carve = [&](size_t bytes) {
        unsigned char* p = cursor;
        cursor += (bytes + 15) & ~(size_t)15;
        return p;
    };
    // FAST: the FP32 production instantiation reads the amplitude from the K1Table rows; the
    // others from the knots and natural-unit coefficients of a SplineView
    constexpr bool FAST = sizeof(TF) == sizeof(float) && !KC;
    double* x64 = reinterpret_cast<double*>(carve(sizeof(double) * n));
    TF* xf = FAST ? nullptr : reinterpret_cast<TF*>(carve(sizeof(TF) * n));
    TF* cf = FAST ? nullptr : reinterpret_cast<TF*>(carve(sizeof(TF) * 4 * (n - 1)));
    float4* tab = FAST ? reinterpret_cast<float4*>(carve(sizeof(float4) * (n + 1))) : nullptr;
    K1Z<TF>* zt = reinterpret_cast<K1Z<TF>*>(carve(sizeof(K1Z<TF>) * per_split));
    double* zw = reinterpret_cast<double*>(carve(sizeof(double) * per_split));
    K1Z<double>* zd = reinterpret_cast<K1Z<double>*>(carve(sizeof(K1Z<double>) * 16));
    double* zdw = reinterpret_cast<double*>(carve(sizeof(double) * 16));
    __shared__ double warp_sum[kK1Threads / 32];
    __shared__ TF sh2f[24], awf[24];
    const double* src_coef = spline + n;  // log N block
    const double x_knot = spline[knot];
    const double h64 = (spline[n - 1] - spline[0]) / (double)(n - 1);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        x64[i] = spline[i] - x_knot;
        if constexpr (!FAST) xf[i] = (TF)(spline[i] - x_knot);
    }
    if constexpr (FAST) {
        for (int i = threadIdx.x; i < n - 1; i += blockDim.x) {
            const double* c = src_coef + 4 * (size_t)i;
            tab[i + 1] = make_float4((float)c[0], (float)(c[1] * h64), (float)(c[2] * h64 * h64),
                                     (float)(c[3] * h64 * h64 * h64));
        }
        if (threadIdx.x == 0) {
            tab[0] = make_float4(-200.0f, 0.0f, 0.0f, 0.0f);
            tab[n] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    } else {
        for (int i = threadIdx.x; i < 4 * (n - 1); i += blockDim.x) cf[i] = (TF)src_coef[i];
    }
    if (threadIdx.x < 24) {
        sh2f[threadIdx.x] = (TF)consts.sh2[threadIdx.x];
        awf[threadIdx.x] = (TF)consts.aw[threadIdx.x];
    }
    if (threadIdx.x < 16) zdw[threadIdx.x] = 0.0;
    __syncthreads();
    SplineView<double> sd;
    // the FP64 panel nodes read the coefficients from global memory (L1/L2): keeping them
    // out of shared memory lets four CTAs share an SM
    sd.x = x64; sd.coef = src_coef; sd.n = n; sd.x0 = x64[0];
    sd.inv_h = (double)(n - 1) / (x64[n - 1] - x64[0]);
    SplineView<TF> sf;
    if constexpr (!FAST) {
        sf.x = xf; sf.coef = cf; sf.n = n; sf.x0 = xf[0];
        sf.inv_h = (TF)((double)(n - 1) / (x64[n - 1] - x64[0]));
    }
    const double r = r_grid[knot];
    const K1Parent<double> Pd = k1_parent<double>(sd, phd, r, knot);
    K1Parent<TF> Pf;
    K1Table tf;
    if constexpr (FAST) {
        // the parent in FP32 from its FP64 values
        Pf.r = (float)r;
        Pf.lr_abs = (float)::log(r);
        Pf.r2 = Pf.r * Pf.r;
        Pf.alpha_r = alpha_of_log(Pf.lr_abs, phf);
        Pf.knot = knot;
        Pf.pr = (float)Pd.pr;
        Pf.Nr = (float)Pd.Nr;
        Pf.Sr = (float)Pd.Sr;
        tf.rows = tab;
        tf.inv_h = (float)(1.0 / h64);
        tf.knot = (float)knot;
        tf.top = (float)(n - 1);
        if (knot <= n - 2) {
            const double* c = src_coef + 4 * (size_t)knot;
            tf.rk = make_float4(0.0f, (float)(c[1] * h64), (float)(c[2] * h64 * h64), (float)(c[3] * h64 * h64 * h64));
        } else {
            tf.rk = make_float4(-Pf.pr, 0.0f, 0.0f, 0.0f);  // the last knot: above it N = 1
        }
        // interval knot - 1 about its right end (the knot): p(x) - p(x_knot) as a cubic in x - x_knot
        const double* c = src_coef + 4 * (size_t)(knot - 1);
        const double b1 = c[1] + h64 * (2.0 * c[2] + 3.0 * h64 * c[3]);
        const double c1 = c[2] + 3.0 * h64 * c[3];
        tf.rkm1 = make_float4(0.0f, (float)(b1 * h64), (float)(c1 * h64 * h64), (float)(c[3] * h64 * h64 * h64));
    } else {
        Pf = k1_parent<TF>(sf, phf, r, knot);
    }

    // phase 1: per-node data of this CTA's range; the two intervals adjacent to the
    // parent knot (z -> x) are left to the FP64 table, which every CTA of the cluster
    // prepares (16 nodes) so that the FP64 evaluations can be shared among them
    for (int L = threadIdx.x; L < k_count; L += blockDim.x) {
        const int k = k_begin + L;
        const int iv = k >> 3, m = k & 7;
        if (iv == knot - 1 || iv == knot) {
            zw[L] = 0.0;
            continue;
        }
        // node positions from the absolute knots (the reference rule), then relative to log r
        const double xa = spline[iv], xb = spline[iv + 1];
        const double hw = 0.5 * (xb - xa);
        const double lz = 0.5 * (xa + xb) + hw * consts.rule.x8[m];
        const double rw = hw * consts.rule.w8[m];
        if constexpr (FAST)
            zt[L] = k1_prepare_z_fast(tf, Pf, phf, lz - x_knot, lz);
        else
            zt[L] = k1_prepare_z<TF>(sf, Pf, phf, lz - x_knot, lz);
        const double z = (double)zt[L].z;
        zw[L] = 2.0 * z * z * rw;
    }
    if (threadIdx.x < 16) {
        const int iv = knot - 1 + (int)(threadIdx.x >> 3), m = threadIdx.x & 7;
        if (iv >= 0 && iv < n - 1) {
            const double xa = spline[iv], xb = spline[iv + 1];
            const double hw = 0.5 * (xb - xa);
            const double lz = 0.5 * (xa + xb) + hw * consts.rule.x8[m];
            zd[threadIdx.x] = k1_prepare_z<double>(sd, Pd, phd, lz - x_knot, lz);
            zdw[threadIdx.x] = 2.0 * zd[threadIdx.x].z * zd[threadIdx.x].z * (hw * consts.rule.w8[m]);
        }
    }
    __syncthreads();

    double total = 0.0;
    // phase 3 first: the FP64 evaluations of the panel nodes, every kK1Split-th one per CTA, on
    // the last threads (the FP32 sweep below gives them no more items than the others), so that
    // the FP32 warps overlap their FP64 latency instead of idling behind it at the reduction
    for (int e = split + kK1Split * (int)(blockDim.x - 1 - threadIdx.x); e < 16 * 24; e += kK1Split * blockDim.x) {
        const int idx = e / 24, j = e - 24 * (e / 24);
        const double w = zdw[idx];
        if (w != 0.0)
            total += k1_point<double, KC, sizeof(TF) == sizeof(float)>(sd, Pd, zd[idx], phd, consts.sh2[j], history,
                                                                         r_grid) *
                     consts.aw[j] * w;
    }
    // phase 2: the flattened (node, angle) evaluations, an equal share per thread; the
    // mixed build without the constraint takes two angles of a node per step on the
    // packed FP32x2 instructions
    if constexpr (sizeof(TF) == sizeof(float) && !KC) {
        for (int e = threadIdx.x; e < k_count * 12; e += blockDim.x) {
            const int L = e / 12, j = 2 * (e - 12 * L);
            const double w = zw[L];
            if (w != 0.0) {
                const f2 v = k1_pair_point(tf, Pf, zt[L], phf, make_float2(sh2f[j], sh2f[j + 1]));
                total += ((double)(v.x * awf[j]) + (double)(v.y * awf[j + 1])) * w;
            }
        }
    } else {
        for (int e = threadIdx.x; e < k_count * 24; e += blockDim.x) {
            const int L = e / 24, j = e - 24 * (e / 24);
            const double w = zw[L];
            if (w != 0.0)
                total += (double)(k1_point<TF, KC>(sf, Pf, zt[L], phf, sh2f[j], history, r_grid) * awf[j]) * w;
        }
    }
    // deterministic block reduction, then the cluster's partials in rank order
    __shared__ double cta_total;
    for (int o = 16; o > 0; o >>= 1) total += __shfl_down_sync(0xffffffffu, total, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = total;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kK1Threads / 32; ++w) s += warp_sum[w];
        cta_total = s;
    }
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    if (cluster.block_rank() == 0 && threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < kK1Split; ++q) s += *cluster.map_shared_rank(&cta_total, q);
        out[knot] = s;
    }
    cluster.sync();  // keep every CTA's shared memory alive until rank 0 has read it
}

// Per r-grid interval i: the window start max(i-3, 0) (-1 when the 6-point window runs
// past the grid), the local interval, and the rows of the linear maps y -> M_j, M_{j+1}
// of the natural spline through the window (one Thomas solve per unit vector, the
// tridiagonal system of numerics/interpolation.py:13-50).
__global__ void kc_weights_kernel(const double* __restrict__ r, int n, double* __restrict__ weights)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    double* w = weights + (size_t)i * kKcStride;
    const int start = i - 3 < 0 ? 0 : i - 3;
    for (int k = 0; k < kKcStride; ++k) w[k] = 0.0;
    if (start + 6 > n) {
        w[0] = -1.0;
        return;
    }
    const int j = i - start;
    w[0] = start;
    w[1] = j;
    double h[5];
    for (int k = 0; k < 5; ++k) h[k] = r[start + k + 1] - r[start + k];
    for (int e = 0; e < 6; ++e) {
        // right-hand side 6 ((y2-y1)/h1 - (y1-y0)/h0) of unit vector e, interior rows 1..4
        double rhs[4], cp[4], dp[4], M[6];
        for (int q = 0; q < 4; ++q) {
            const double y0 = e == q ? 1.0 : 0.0, y1 = e == q + 1 ? 1.0 : 0.0, y2 = e == q + 2 ? 1.0 : 0.0;
            rhs[q] = 6.0 * ((y2 - y1) / h[q + 1] - (y1 - y0) / h[q]);
        }
        for (int q = 0; q < 4; ++q) {
            const double diag = 2.0 * (h[q] + h[q + 1]);
            const double sub = q > 0 ? h[q] : 0.0;
            const double den = diag - (q > 0 ? sub * cp[q - 1] : 0.0);
            cp[q] = q < 3 ? h[q + 1] / den : 0.0;
            dp[q] = (rhs[q] - (q > 0 ? sub * dp[q - 1] : 0.0)) / den;
        }
        M[0] = 0.0;
        M[5] = 0.0;
        M[4] = dp[3];
        for (int q = 2; q >= 0; --q) M[q + 1] = dp[q] - cp[q] * M[q + 2];
        w[2 + e] = M[j];
        w[8 + e] = M[j + 1];
    }
}

}  // namespace

cudaError_t launch_kc_weights(const double* r, int points, double* weights, cudaStream_t stream)
{
    kc_weights_kernel<<<(points + 127) / 128, 128, 0, stream>>>(r, points, weights);
    return cudaGetLastError();
}

cudaError_t launch_k1(const nlo_bk_params& p, const double* r, int points, const double* spline,
                      const int32_t* active, const int32_t* count, double* out, cudaStream_t stream,
                      const K1History& history, int sets)
{
    if (history.on && sets != 1) return cudaErrorInvalidValue;
    K1Consts consts;
    consts.rule = k1_rule();
    for (int j = 0; j < 24; ++j) {
        const double v = 0.5 * (consts.rule.x24[j] + 1.0);
        const double theta = kPi * v * v;
        const double sh = std::sin(0.5 * theta);
        consts.sh2[j] = sh * sh;
        consts.aw[j] = consts.rule.w24[j] * kPi * v;
    }
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * (size_t)points * sets, stream);
    if (e != cudaSuccess) return e;
    const Phys<double> phd = make_phys<double>(p);
    const size_t per_split = (size_t)((points - 1 + kK1Split - 1) / kK1Split) * 8;
    // the carve order of k1_kernel: x64, then the knots and coefficients (or, in the FP32
    // production instantiation, the K1Table rows), the node tables
    auto smem_for = [&](size_t tf, bool fast) {
        auto a16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
        const size_t amplitude = fast ? a16(sizeof(float4) * (size_t)(points + 1))
                                      : a16(tf * (size_t)points) + a16(tf * 4 * (size_t)(points - 1));
        return a16(8 * (size_t)points) + amplitude +
               a16((tf == 4 ? sizeof(K1Z<float>) : sizeof(K1Z<double>)) * per_split) + a16(8 * per_split) +
               a16(sizeof(K1Z<double>) * 16) + a16(8 * 16);
    };
    auto launch = [&](auto tag, auto kc) -> cudaError_t {
        using TF = decltype(tag);
        constexpr bool KC = decltype(kc)::value;
        const size_t smem = smem_for(sizeof(TF), sizeof(TF) == sizeof(float) && !KC);
        const void* fn = (const void*)k1_kernel<TF, KC>;
        cudaError_t err = raise_dynamic_smem(fn, smem);
        if (err == cudaSuccess) err = prefer_shared_carveout(fn);
        if (err != cudaSuccess) return err;
        k1_kernel<TF, KC><<<dim3(points, kK1Split, sets), kK1Threads, smem, stream>>>(make_phys<TF>(p), phd, consts, history,
                                                                               r, points, spline, active, count, out);
        return cudaGetLastError();
    };
    using On = std::true_type;
    using Off = std::false_type;
    if (p.precision == NLO_PRECISION_FP64)
        return history.on ? launch(double(), On()) : launch(double(), Off());
    return history.on ? launch(float(), On()) : launch(float(), Off());
}

}  // namespace nlo
