// The K2 + Kf integrand of the BK right-hand side in its cancellation-free form, shared by
// the quasi-Monte Carlo kernel (k2kf.cu) and the Vegas kernel (k2kf_vegas.cu):
// _nlo_integrand x exp(2 log z + 2 log z') of bk/derivatives.py:322-335 and 490-612, with
// the kernels of bk_kernels/k2.py:8-39 and bk_kernels/kf.py:10-41.  A sample's
// parent-independent quantities (z, z', |z - z'|, their amplitudes, the Jacobian) form a
// record (k2_prepare*); k2_point evaluates one (record, parent) pair.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "sobol.cuh"

namespace nlo {
namespace k2 {

// Per-sample record (r-independent), 20 values.
enum Rec {
    kZ, kZ2, kS1, kS2, kP1, kP2, kU1, kV1, kU2, kV2,
    kQ, kD1, kD2, kDN, kSY, kLmin, kCpt, kDl, kZsq, kZ2sq,
    kRecLen
};

template <typename T>
struct alignas(16) K2Rec {
    T v[kRecLen];
};

template <typename T>
struct K2Box {
    T lower[4], width[4];
    T cpt_scale;  // volume * Nc^2 / (8 pi^4)
};

// atanh(t)/t - 1 = t^2 g(t^2), g(x) = sum_{k>=0} x^k/(2k+3), for t^2 < 1/4: the series in
// FP64; the FP32 pair path (k2_pair_fast) evaluates g by a degree-6 polynomial fitted on
// [0, 1/4] in relative error (least squares at Chebyshev nodes; 8e-8 relative in FP32
// Horner, i.e. FP32 rounding).
template <typename T>
__device__ __forceinline__ T atanh_ratio_m1(T t2);

template <>
__device__ __forceinline__ double atanh_ratio_m1<double>(double t2)
{
    double s = 0.0;
#pragma unroll
    for (int k = 30; k >= 1; --k) s = fma(s, t2, 1.0 / (2.0 * k + 1.0));
    return s * t2;
}

template <>
__device__ __forceinline__ float atanh_ratio_m1<float>(float t2)
{
    float g = fmaf(0.15609439065092748f, t2, 0.04106302733766397f);
    g = fmaf(g, t2, 0.09747851219255123f);
    g = fmaf(g, t2, 0.11051354325642386f);
    g = fmaf(g, t2, 0.1428825580061165f);
    g = fmaf(g, t2, 0.19999959971627077f);
    g = fmaf(g, t2, 0.33333333435159396f);
    return g * t2;
}

// The parent-independent record of one sample at box coordinates x = (log z, log z',
// theta_z, theta_z'); `valid` false gives a record of zero weight.
template <typename T>
__device__ __forceinline__ void k2_prepare_x(const SplineView<T>& s, const K2Box<T>& box, const T* x, bool valid,
                                             T* rec)
{
    const T lz = x[0], lz2 = x[1], th = x[2], th2 = x[3];
    const T z = M<T>::exp_acc(lz), z2 = M<T>::exp_acc(lz2);
    const T sh1 = M<T>::sin((T)0.5 * th), sh2 = M<T>::sin((T)0.5 * th2);
    const T c1 = M<T>::cos(th), c2 = M<T>::cos(th2);
    const T dth = th - th2;
    const T c12 = M<T>::cos(dth), sh12 = M<T>::sin((T)0.5 * dth);
    const T zzsq = (z - z2) * (z - z2) + (T)4 * z * z2 * sh12 * sh12;
    valid = valid && zzsq >= M<T>::tiny_square();
    const T lzz = (T)0.5 * M<T>::log_acc(zzsq);
    const NS<T> Y = eval_s_log(s, lz), Y2 = eval_s_log(s, lz2), ZZ = eval_s_log(s, lzz);
    const T dN = ndiff_s(Y2, Y);  // N_Y2 - N_Y
    rec[kZ] = z;
    rec[kZ2] = z2;
    rec[kS1] = z * (sh1 * sh1);  // z sin^2(theta/2): X^2 = (r - z)^2 + 4 r rec[kS1]
    rec[kS2] = z2 * (sh2 * sh2);
    rec[kP1] = (z2 - z) * (z2 + z);
    rec[kP2] = (T)2 * z * z2 * (z2 * c1 - z * c2);
    rec[kU1] = z2 - z * c12;
    rec[kV1] = z * (z * c2 - z2 * c1);
    rec[kU2] = z - z2 * c12;
    rec[kV2] = z2 * (z2 * c1 - z * c2);
    rec[kQ] = valid ? M<T>::rcp(zzsq) : (T)0;
    // S_Y - S_zz S_Y2 = S_Y N_zz + S_zz (N_Y2 - N_Y);  S_Y2 - S_zz S_Y = S_Y2 N_zz - S_zz (N_Y2 - N_Y)
    rec[kD1] = Y.S * ZZ.N + ZZ.S * dN;
    rec[kD2] = Y2.S * ZZ.N - ZZ.S * dN;
    rec[kDN] = dN;
    rec[kSY] = Y.S;
    rec[kLmin] = M<T>::fmin(M<T>::fmin(lz, lz2), lzz);
    rec[kCpt] = valid ? box.cpt_scale * M<T>::exp_acc((T)2 * lz + (T)2 * lz2) : (T)0;
    rec[kDl] = (T)2 * (lz2 - lz);
    rec[kZsq] = z * z;
    rec[kZ2sq] = z2 * z2;
}

template <typename T>
struct K2Parent {
    T r, r2, lr, two_r;
    T alpha_r;  // the RC_NLO = PARENT_NLO coupling
};

// K2 and Kf contributions of one sample to one parent (already weighted).
template <typename T, bool SYM, typename EvalSpline>
__device__ __forceinline__ void k2_point(const EvalSpline& s, const Phys<T>& ph, const K2Parent<T>& P,
                                         const T* __restrict__ rec, T& k2w, T& kfw)
{
    const T r = P.r;
    const T z = rec[kZ], z2 = rec[kZ2];
    const T Xsq = (r - z) * (r - z) + (T)4 * r * rec[kS1];
    const T X2sq = (r - z2) * (r - z2) + (T)4 * r * rec[kS2];
    const bool valid = Xsq >= M<T>::tiny_square() && X2sq >= M<T>::tiny_square();
    const T lXs = M<T>::log_fast(Xsq), lX2s = M<T>::log_fast(X2sq);
    const PS<T> vX = eval_s_ps(s, (T)0.5 * lXs), vX2 = eval_s_ps(s, (T)0.5 * lX2s);
    // kernels (k2.py, kf.py) in the stable form
    const T a = Xsq * rec[kZ2sq], b = X2sq * rec[kZsq];
    const T sab = a + b;
    const T rs = M<T>::rcp(sab);
    const T d = r * (r * rec[kP1] - rec[kP2]);
    const T t = d * rs;
    const T t2 = t * t;
    T hm1, Ld;
    if (t2 < (T)0.25) {
        hm1 = atanh_ratio_m1<T>(t2);
        Ld = (T)2 * t * ((T)1 + hm1);
    } else {
        Ld = lXs - lX2s + rec[kDl];  // log(a/b)
        hm1 = M<T>::div(Ld, (T)2 * t) - (T)1;
    }
    const T q = rec[kQ];
    const T L = (T)2 * ((T)1 + hm1) * rs;
    const T f = (T)2 * hm1;
    const T fq2 = f * q * q;
    const T r2Lq = P.r2 * L * q;
    const T C0 = fq2 - (T)4 * r2Lq;
    // L r^4/a + log(a/b) r^2 q/a = L r^2 q 2 r B1/(X^2 z'), B1 = r (z' - z c12) + z (z c2 - z' c1)
    const T B1 = r * rec[kU1] + rec[kV1];
    const T B2 = r * rec[kU2] + rec[kV2];
    T k2 = C0 + r2Lq * P.two_r * B1 * M<T>::rcp(Xsq * z2);
    T k2s = C0 + r2Lq * P.two_r * B2 * M<T>::rcp(X2sq * z);
    const T kf = (r2Lq - fq2) * ph.nf_over_nc;
    T dip = vX.S * rec[kD1];
    T dips = vX2.S * rec[kD2];
    if (M<T>::fabs(k2) > (T)1e10 && M<T>::fabs(dip) < (T)1e-10) { k2 = (T)0; dip = (T)0; }
    if (M<T>::fabs(k2s) > (T)1e10 && M<T>::fabs(dips) < (T)1e-10) { k2s = (T)0; dips = (T)0; }
    const T dNX = ndiff_ps(vX, vX2);
    T k2part, fermion;
    if (SYM) {
        k2part = (T)0.5 * (k2 * dip + k2s * dips);
        fermion = (T)0.5 * kf * dNX * rec[kDN];
    } else {
        k2part = k2 * dip;
        fermion = kf * rec[kSY] * dNX;
    }
    if (!(ph.nf > (T)0)) fermion = (T)0;
    const T lmin = M<T>::fmin(M<T>::fmin(rec[kLmin], P.lr), (T)0.5 * M<T>::fmin(lXs, lX2s));
    // _nlo_alpha_s (bk/derivatives.py:615-632): the smallest of the six sizes, or the parent
    const T alpha = ph.nlo_parent ? P.alpha_r : alpha_of_log(lmin, ph);
    const T scale = alpha * alpha * rec[kCpt];
    k2w = k2part * scale;
    kfw = -fermion * scale;
    if (!valid || !M<T>::finite(k2w)) k2w = (T)0;
    if (!valid || !M<T>::finite(kfw)) kfw = (T)0;
}

// The record of Sobol point `index` mapped into the box (explicitly rounded operations, as
// the oracle replays them).
template <typename T>
__device__ __forceinline__ void k2_prepare(const SplineView<T>& s, const K2Box<T>& box, const uint32_t* state,
                                           const uint32_t* shift, uint64_t index, bool valid, T* rec)
{
    T x[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        const T u = sobol_unit<T>(sobol_bits(state + 30 * d, shift[d], index), index);
        x[d] = M<T>::add_rn(box.lower[d], M<T>::mul_rn(box.width[d], u));
    }
    k2_prepare_x<T>(s, box, x, valid, rec);
}

}  // namespace k2
}  // namespace nlo
