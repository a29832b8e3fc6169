// NLO DIS integrands on the unit cube (dis/observables.py:107-331, dis/lo.py,
// dis/transverse.py, dis/longitudinal.py).
//
// Each term maps a unit-cube point x to the physical variables, evaluates the impact
// factor and multiplies by the dipole amplitude, the coupling and the Jacobian exactly as
// the reference's integrand_* functions do.  The map and every "1 - something" /
// squared-distance that can cancel are formed in FP64 (they are a few dozen operations
// per sample); the impact-factor bodies -- the Bessel functions, logarithms and the long
// polynomial combinations -- run in the arithmetic type T.  The bodies restate the
// reference's expressions term by term; where the reference writes 1 - z, 1 + gamma - 2 z
// or the argument of Li2, the code uses the exact complements formed in FP64 so that FP32
// does not lose the small differences near the end points.
#pragma once

#include "dis_math.cuh"
#include "dis_table.cuh"

namespace nlo {
namespace dis {

enum Term : int {
    kTermLO = 0,
    kTermDip0 = 1,  // T0 / Omega_L_const   (2D)
    kTermDip1 = 2,  // T1 / ab              (3D)
    kTermDip2 = 3,  // T2 / cd              (4D)
    kTermI1 = 4,    // qg I1                (5D)
    kTermI2 = 5,    // qg I2, y_t explicit  (6D)
    kTermI3 = 6,    // qg I3, y_t1, y_t2    (7D)
    kTermI2N = 7,   // qg I2, inner rule    (5D)
    kTermI3N = 8,   // qg I3, inner rule    (5D)
    kTermCount = 9,
};

__host__ __device__ constexpr int term_dims(int term)
{
    return term == kTermLO || term == kTermDip0 ? 2
         : term == kTermDip1                    ? 3
         : term == kTermDip2                    ? 4
         : term == kTermI2                      ? 6
         : term == kTermI3                      ? 7
                                                : 5;
}

constexpr int kMaxQuarks = 8;
constexpr int kMaxInner = 128;

struct InnerRule {
    int n;
    double y[kMaxInner];
    double w[kMaxInner];
};

// Everything a term needs, fixed per (Q^2, x_Bj, quark, polarisation) job.
template <typename T>
struct DisArgs {
    double Q2, xbj, mf, maxr;
    double Ydip;        // rapidity of the dipole terms (dis/observables.py:62-76)
    double Ylo;         // max(log(X0/x_Bj), 0) of the LO term (dis/lo.py:49)
    double z2min, W2;   // qg: Q0^2/W^2 and W^2 = Q^2/x_Bj (dis/observables.py:56-85)
    double gm1;         // gamma - 1 with gamma = sqrt(1 + 4 m^2/Q^2)
    int n_quarks;
    double lo_mass[kMaxQuarks], lo_e2[kMaxQuarks];
    bool transverse, finite_nc, parent_coupling;
    Coupling<T> coup;
    // dipole
    bool table;
    GBWParams<T> gbw;
    double gbw_min_r, gbw_max_r;
    TableView tab;
};

template <typename T>
__device__ __forceinline__ T amplitude(const DisArgs<T>& a, double r, double Y)
{
    if (a.table) return (T)table_amplitude(a.tab, r, Y);
    return gbw_amplitude(a.gbw, (T)r, (T)Y);
}

// The three dipoles of a qg sample at one rapidity: a table looks its rows up once.
template <typename T>
__device__ __forceinline__ void amplitudes3(const DisArgs<T>& a, double r01, double r02, double r21, double Y, T& N01,
                                            T& N02, T& N21)
{
    if (a.table) {
        const TableRow row = table_row(a.tab, Y);
        N01 = (T)table_amplitude_at(a.tab, row, r01);
        N02 = (T)table_amplitude_at(a.tab, row, r02);
        N21 = (T)table_amplitude_at(a.tab, row, r21);
    } else {
        N01 = gbw_amplitude(a.gbw, (T)r01, (T)Y);
        N02 = gbw_amplitude(a.gbw, (T)r02, (T)Y);
        N21 = gbw_amplitude(a.gbw, (T)r21, (T)Y);
    }
}

template <typename T>
__device__ __forceinline__ double dipole_min_r(const DisArgs<T>& a)
{
    return a.table ? a.tab.hdr[kHdrRmin] : a.gbw_min_r;
}

template <typename T>
__device__ __forceinline__ double dipole_max_r(const DisArgs<T>& a)
{
    return a.table ? a.tab.hdr[kHdrRmax] : a.gbw_max_r;
}

template <typename T>
__device__ __forceinline__ T alpha_bar(const DisArgs<T>& a, T r)
{
    return alpha_s(a.coup, r) * (T)(kCF / kPi);
}

// ===========================================================================
// LO: sum_q e_q^2 |Psi|^2 N(r, Y) 2 pi r maxr   (dis/lo.py:22-49, dis/observables.py:352-359)
template <typename T>
__device__ T lo_term(const DisArgs<T>& a, const double* x)
{
    const double z = x[0], zb = 1.0 - x[0];
    const double r = a.maxr * x[1];
    T total = 0;
    for (int q = 0; q < a.n_quarks; ++q) {
        const double mf = a.lo_mass[q];
        const T eps = DM<T>::sqrt((T)(a.Q2 * z * zb + mf * mf));
        const T arg = (T)r * eps;
        if (!(arg >= (T)1e-7 && arg <= (T)5e2)) continue;
        const K01<T> k = bessel_k01(arg);
        T v;
        if (a.transverse) {
            const T zt = (T)z;
            const T f = (T)1 - (T)2 * zt + (T)2 * zt * zt;
            const T mk = (T)mf * k.k0;
            v = f * eps * eps * k.k1 * k.k1 + mk * mk;
        } else {
            const T zz = (T)(z * zb);
            v = (T)(4.0 * a.Q2) * zz * zz * k.k0 * k.k0;
        }
        total += (T)a.lo_e2[q] * v;
    }
    const T N = amplitude(a, r, a.Ylo);
    return (T)(2.0 * kPi * r * a.maxr) * total * N;
}

// ===========================================================================
// Virtual (dipole) terms.
template <typename T>
struct DipPoint {
    T z, zb, r, Q2, m2;
    T kz;  // sqrt(z zb Q^2 + m^2)
    T gm1, gam;
};

// (1 + 1/(2z)) core and friends: core(z) = log(1-z) + gamma log((1+gamma)/(1+gamma-2z))
// with 1 + gamma - 2z = (gamma - 1) + 2(1 - z)
template <typename T>
__device__ __forceinline__ T omega_core(const DipPoint<T>& p, T zz, T zzb)
{
    return DM<T>::log(zzb) + p.gam * DM<T>::log(((T)2 + p.gm1) / (p.gm1 + (T)2 * zzb));
}

template <typename T>
__device__ __forceinline__ T log_mass_ratio(const DipPoint<T>& p, T zz, T zzb)
{
    return DM<T>::log1p(zz * zzb * p.Q2 / p.m2);
}

// OmegaT_V (dis/transverse.py:46-61)
template <typename T>
__device__ T omega_t_v(const DipPoint<T>& p)
{
    const T m2q = p.m2 / p.Q2;
    T total = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const T zz = s == 0 ? p.z : p.zb;
        const T zzb = s == 0 ? p.zb : p.z;
        const T inv2z = (T)0.5 / zz;
        total += ((T)1 + inv2z) * omega_core(p, zz, zzb)
               - inv2z * ((zz + (T)0.5) * (-p.gm1) + m2q) * log_mass_ratio(p, zz, zzb);
    }
    return total;
}

// OmegaT_N (dis/transverse.py:64-75); 1 + z - 2 z^2 = (1 - z)(1 + 2 z)
template <typename T>
__device__ T omega_t_n(const DipPoint<T>& p)
{
    const T m2q = p.m2 / p.Q2;
    T out = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const T zz = s == 0 ? p.z : p.zb;
        const T zzb = s == 0 ? p.zb : p.z;
        const T v = zzb * ((T)1 + (T)2 * zz) / zz * omega_core(p, zz, zzb)
                  + zzb / zz * (((T)0.5 + zz) * p.gm1 - m2q) * log_mass_ratio(p, zz, zzb);
        out += s == 0 ? v : -v;
    }
    return out;
}

// OmegaL_V (dis/longitudinal.py:130-143)
template <typename T>
__device__ T omega_l_v(const DipPoint<T>& p)
{
    return (T)0.5 / p.z * omega_core(p, p.z, p.zb) + (T)0.5 / p.zb * omega_core(p, p.zb, p.z)
         + (T)0.25 / (p.z * p.zb) * (p.gm1 + (T)2 * p.m2 / p.Q2) * log_mass_ratio(p, p.z, p.zb);
}

// L_dip (dis/longitudinal.py:146-156).  With g = gamma - 1:
//   1/(1 - (1-gamma)/(2z)) = 2z/(2z + g),   1/(1 - (1+gamma)/(2z)) = -2z/(2(1-z) + g)
template <typename T>
__device__ T l_dip(const DipPoint<T>& p, T lz)
{
    T total = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const T zz = s == 0 ? p.z : p.zb;
        const T zzb = s == 0 ? p.zb : p.z;
        total += li2((T)2 * zz / ((T)2 * zz + p.gm1)) + li2(-(T)2 * zz / ((T)2 * zzb + p.gm1));
    }
    return total - ((T)kPi2Over6 - (T)0.5 * lz * lz);
}

template <typename T>
__device__ T t_dip0(const DipPoint<T>& p)
{
    const T lz = DM<T>::log(p.z / p.zb);
    const T common = -(T)kPi2Over6 + (T)0.5 * lz * lz + omega_t_v(p) + l_dip(p, lz);
    const K01<T> k = bessel_k01(p.r * p.kz);
    const T a = p.kz * k.k1;
    const T b = DM<T>::sqrt(p.m2) * k.k0;
    return a * a * ((p.z * p.z + p.zb * p.zb) * ((T)2.5 + common) + (p.z - p.zb) * (T)0.5 * omega_t_n(p))
         + b * b * ((T)3 + common);
}

template <typename T>
__device__ __forceinline__ T xi_factor(T xi, T xib, T lxi)
{
    return ((T)2 * lxi / xib - ((T)1 + xi) * (T)0.5) / xi;
}

// T1 (dis/transverse.py:78-142)
template <typename T>
__device__ T t_dip1(const DipPoint<T>& p, T xi, T xib)
{
    const K01<T> kz = bessel_k01(p.r * p.kz);
    const T lxi = DM<T>::log(xi);
    const T xf = xi_factor(xi, xib, lxi);
    T v1 = 0, vms1 = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const T zz = s == 0 ? p.z : p.zb;
        const T zzb = s == 0 ? p.zb : p.z;
        const T sh = DM<T>::sqrt(p.kz * p.kz + xi / xib * zzb * p.m2);
        const K01<T> ks = bessel_k01(p.r * sh);
        v1 += xf * (sh * ks.k1 - p.kz * kz.k1)
            - (lxi / (xib * xib) + zz / xib + zz * (T)0.5) * zzb * p.m2 / sh * ks.k1;
        vms1 += xf * (ks.k0 - kz.k0) + (-(T)1.5 * zzb / xib + zzb * (T)0.5) * ks.k0;
    }
    return p.kz * kz.k1 * (p.z * p.z + p.zb * p.zb) * v1 + p.m2 * kz.k0 * vms1;
}

// sqrt(kb^2 + d) K1(r sqrt(.)) - kb K1(r kb), linearised below 1e-5 relative
// (dis/transverse.py:13-23)
template <typename T>
__device__ __forceinline__ T weighted_k1_difference(T r, T kb, T d, const K01<T>& kbase)
{
    const T b2 = kb * kb;
    const T s2 = b2 + d;
    if (!(s2 > (T)0 && kb > (T)0)) return (T)0;
    const T rel = fabs(d) / (b2 + fabs(d) + (T)(sizeof(T) == 8 ? 1e-300 : 1e-37));
    if (rel < (T)1e-5) return -(T)0.5 * r * d * kbase.k0;
    const T sh = DM<T>::sqrt(s2);
    return sh * bessel_k1(r * sh) - kb * kbase.k1;
}

template <typename T>
struct T2Side {
    T v2, vms2, n;
};

// V2 / VMS2 / N unsymmetric pieces (dis/transverse.py:168-300) at fraction zz
template <typename T>
__device__ T2Side<T> t2_side(const DipPoint<T>& p, T zz, T zzb, T chi, T chib, T u, const K01<T>& kz)
{
    const T m2 = p.m2;
    const T kc2 = chi * chib * p.Q2 + m2;
    const T d = u * zzb / chib * kc2;
    const T sh = DM<T>::sqrt(p.kz * p.kz + d);
    const K01<T> ks = bessel_k01(p.r * sh);
    const T uu = u / (u + (T)1);
    const T up1 = u + (T)1;
    const T zc = zz - chi;
    T2Side<T> o;
    o.v2 = -(T)1 / chib / (u * up1) * m2 / kc2 * ((T)2 * chi + uu * uu / zz * zc * ((T)1 - (T)2 * chi))
               * weighted_k1_difference(p.r, p.kz, d, kz)
         - (T)1 / (chib * chib) / up1 * zc * ((T)1 - (T)2 * uu * zc + uu * uu / zz * zc * zc) * m2 / sh * ks.k1;
    o.vms2 = (T)1 / chib / (up1 * up1) * (-zz - uu * (zz + u * chi) / zz * (chi - zzb)) * ks.k0
           + (T)1 / (up1 * up1 * up1)
                 * (p.kz * p.kz / kc2 * ((T)1 + u * chi * chib / (zz * zzb))
                    - m2 / kc2 * chi / chib * ((T)2 * up1 * up1 / u + u / (zz * zzb) * zc * zc))
                 * (ks.k0 - kz.k0);
    const T pref = (T)2 * zzb / zz / (up1 * up1 * up1);
    o.n = pref * (((T)2 + u) * u * zz + u * u * chi) * sh * ks.k1
        + pref * m2 / kc2 * (zz / zzb + chi / chib * (u - (T)2 * zz - (T)2 * u * chi)) * (sh * ks.k1 - p.kz * kz.k1);
    return o;
}

// ===========================================================================
// Longitudinal dipole terms (dis/longitudinal.py:12-127)
template <typename T>
__device__ T l_omega_const(const DipPoint<T>& p)
{
    const T arg = p.kz * p.r;
    if (!(arg >= (T)1e-7)) return (T)0;
    const T zz = p.z * p.zb;
    const T lz = DM<T>::log(p.z / p.zb);
    const T k0 = bessel_k0(arg);
    return (T)4 * p.Q2 * zz * zz * k0 * k0
         * ((T)2.5 - (T)kPi2Over6 + (T)0.5 * lz * lz + omega_l_v(p) + l_dip(p, lz));
}

template <typename T>
__device__ T l_ab(const DipPoint<T>& p, T xi, T xib)
{
    const T zz = p.z * p.zb;
    const T kz2 = p.kz * p.kz;
    const T b1 = bessel_k0(p.kz * p.r);
    const T b2 = bessel_k0(DM<T>::sqrt(kz2 + p.zb * xi / xib * p.m2) * p.r);
    const T b3 = bessel_k0(DM<T>::sqrt(kz2 + p.z * xi / xib * p.m2) * p.r);
    return (T)4 * p.Q2 * zz * zz * b1 / xi * (-(T)2 * DM<T>::log(xi) / xib + ((T)1 + xi) * (T)0.5)
         * ((T)2 * b1 - b2 - b3);
}

template <typename T>
__device__ T l_cd(const DipPoint<T>& p, T xi, T xib, T x, T xb)
{
    const T arg = p.kz * p.r;
    if (!(arg >= (T)1e-7)) return (T)0;
    const T zz = p.z * p.zb;
    const T kz2 = p.kz * p.kz;
    const T b1 = bessel_k0(arg);
    T total = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const T za = s == 0 ? p.z : p.zb;
        const T zb = s == 0 ? p.zb : p.z;
        const T den = x * xib + xi / zb;
        const T clm = za * za * xib / zb * (-xi * xi + x * xib * ((T)1 + xib * ((T)1 + za * xi / zb)) / den);
        const T kap = xi * p.m2 / (xib * xb * den) * (xi * xb + x * ((T)1 - za * xib / zb));
        total += (b1 - bessel_k0(p.r * DM<T>::sqrt(kz2 / xb + kap))) * clm / (xib * xb * den * (x / xb * kz2 + kap));
    }
    return (T)4 * p.Q2 * zz * zz * b1 * p.m2 * total;
}

// integrand_dip_massive (dis/observables.py:107-172)
template <typename T, int ORDER>
__device__ T dip_term(const DisArgs<T>& a, const double* x)
{
    const double z1 = kZmin + x[0] * (1.0 - 2.0 * kZmin);
    const double z1b = 1.0 - z1;
    const double x01 = a.maxr * x[1];
    const double rmin = dipole_min_r(a), rmax = dipole_max_r(a);
    if (!(x01 >= rmin && x01 <= rmax)) return (T)0;
    const double r = x01;
    DipPoint<T> p;
    p.z = (T)z1;
    p.zb = (T)z1b;
    p.r = (T)r;
    p.Q2 = (T)a.Q2;
    p.m2 = (T)(a.mf * a.mf);
    p.kz = (T)::sqrt(z1 * z1b * a.Q2 + a.mf * a.mf);
    p.gm1 = (T)a.gm1;
    p.gam = (T)(1.0 + a.gm1);
    const T N01 = amplitude(a, r, a.Ydip);
    T v;
    if (a.transverse) {
        if constexpr (ORDER == 0) {
            v = t_dip0(p);
        } else if constexpr (ORDER == 1) {
            v = t_dip1(p, (T)x[2], (T)(1.0 - x[2]));
        } else {
            const K01<T> kz = bessel_k01(p.r * p.kz);
            const double u = (1.0 - x[3]) / x[3];
            T2Side<T> s0, s1;
            {
                const double chi = z1 * x[2];
                s0 = t2_side(p, p.z, p.zb, (T)chi, (T)(1.0 - chi), (T)u, kz);
            }
            {
                const double chi = z1b * x[2];
                s1 = t2_side(p, p.zb, p.z, (T)chi, (T)(1.0 - chi), (T)u, kz);
            }
            const T pre0 = p.z / (T)(x[3] * x[3]);
            const T pre1 = p.zb / (T)(x[3] * x[3]);
            const T v2 = pre0 * s0.v2 + pre1 * s1.v2;
            const T vms2 = pre0 * s0.vms2 + pre1 * s1.vms2;
            const T n = pre0 * s0.n - pre1 * s1.n;
            v = p.kz * kz.k1 * ((p.z * p.z + p.zb * p.zb) * v2 + (p.z - p.zb) * (T)0.5 * n) + p.m2 * kz.k0 * vms2;
        }
    } else {
        if constexpr (ORDER == 0)
            v = l_omega_const(p);
        else if constexpr (ORDER == 1)
            v = l_ab(p, (T)x[2], (T)(1.0 - x[2]));
        else
            v = l_cd(p, (T)x[2], (T)(1.0 - x[2]), (T)x[3], (T)(1.0 - x[3]));
    }
    const T out = N01 * v * (T)(x01 * a.maxr * (1.0 - 2.0 * kZmin)) * alpha_bar(a, p.r);
    return DM<T>::finite(out) ? out : (T)0;
}

// ===========================================================================
// qqbar-g terms.  Side 0 ("j" in dis/transverse.py, "k" in dis/longitudinal.py) pairs
// the gluon with the quark at x0, side 1 with the antiquark at x1.
template <typename T>
struct Trip {
    T z0, z1, z2;
    T zj, zk;        // z0 + z2, z1 + z2
    T m2, Q2;
    T x20x21;
    T Qb2[2], omega[2], lam[2], x2sq[2], x3sq[2];
    T x2jx3j, x2kx3k, x2jx3k, x2kx3j, x3jx3k;
};

// _tripole_variables (dis/transverse.py:937-1000), formed in FP64
template <typename T>
__device__ __forceinline__ Trip<T> make_trip(double Q2, double mf, double z1, double z2, double x01sq, double x02sq,
                                             double x21sq)
{
    const double z0 = 1.0 - z1 - z2;
    const double x20x21 = -0.5 * (x01sq - x21sq - x02sq);
    const double fj = z0 / (z0 + z2), fk = z1 / (z1 + z2);
    Trip<T> t;
    t.z0 = (T)z0;
    t.z1 = (T)z1;
    t.z2 = (T)z2;
    t.zj = (T)(z0 + z2);
    t.zk = (T)(z1 + z2);
    t.m2 = (T)(mf * mf);
    t.Q2 = (T)Q2;
    t.x20x21 = (T)x20x21;
    t.Qb2[0] = (T)(Q2 * z1 * (1.0 - z1));
    t.Qb2[1] = (T)(Q2 * z0 * (1.0 - z0));
    t.omega[0] = (T)(z0 * z2 / (z1 * (z0 + z2) * (z0 + z2)));
    t.omega[1] = (T)(z1 * z2 / (z0 * (z1 + z2) * (z1 + z2)));
    t.lam[0] = (T)(z1 * z2 / z0);
    t.lam[1] = (T)(z0 * z2 / z1);
    t.x2sq[0] = (T)x02sq;
    t.x2sq[1] = (T)x21sq;
    t.x3sq[0] = (T)(fj * fj * x02sq + x21sq - 2.0 * fj * x20x21);
    t.x3sq[1] = (T)(fk * fk * x21sq + x02sq - 2.0 * fk * x20x21);
    t.x2jx3j = (T)(x20x21 - fj * x02sq);
    t.x2kx3k = (T)(-x20x21 + fk * x21sq);
    t.x2jx3k = (T)(-x02sq + fk * x20x21);
    t.x2kx3j = (T)(x21sq - fj * x20x21);
    t.x3jx3k = (T)(fj * x02sq + fk * x21sq - (1.0 + fj * fk) * x20x21);
    return t;
}

template <typename T>
__device__ __forceinline__ T side_P(const Trip<T>& t, int s)
{
    const T za = s == 0 ? t.z0 : t.z1;
    const T zs = s == 0 ? t.zj : t.zk;
    return ((T)2 * za * zs + t.z2 * t.z2) / (zs * zs);
}

template <typename T>
__device__ __forceinline__ T side_A(const Trip<T>& t, int s)
{
    const T zb = s == 0 ? t.z1 : t.z0;
    return (T)1 - (T)2 * zb * ((T)1 - zb);
}

template <typename T>
__device__ __forceinline__ T side_X2(const Trip<T>& t, int s)
{
    return t.x3sq[s] + t.omega[s] * t.x2sq[s];
}

// G22_sing, G12_sing, H (dis/transverse.py:1003-1033) and the Bessel pair at sqrt(M2 X2)
template <typename T>
struct SideSing {
    T k0, k1;  // at sqrt(M2 X2), M2 = Qbar^2 + m^2
    T g22, g12, h;
};

template <typename T>
__device__ __forceinline__ SideSing<T> side_sing(const Trip<T>& t, int s)
{
    const T M2 = t.Qb2[s] + t.m2;
    const T X2 = side_X2(t, s);
    const K01<T> k = bessel_k01(DM<T>::sqrt(M2 * X2));
    const T Mh2 = t.Qb2[s] + t.m2 * ((T)1 + t.lam[s]);
    const K01<T> kh = bessel_k01(DM<T>::sqrt(Mh2 * X2));
    SideSing<T> o;
    o.k0 = k.k0;
    o.k1 = k.k1;
    o.g22 = DM<T>::sqrt(M2 / X2) * k.k1 / t.x2sq[s];
    o.g12 = k.k0 / t.x2sq[s];
    o.h = (T)4 * DM<T>::sqrt(Mh2 / X2) * kh.k1;
    return o;
}

template <typename T>
__device__ __forceinline__ T f_bracket(const Trip<T>& t)
{
    const T z0 = t.z0, z1 = t.z1, z2 = t.z2;
    return z2 * (z0 - z1) * (z0 - z1) * (t.x2jx3j * t.x2kx3k - t.x2kx3j * t.x2jx3k)
         - (z1 * t.zj + z0 * t.zk) * (z0 * t.zj + z1 * t.zk) * t.x20x21 * t.x3jx3k;
}

// transverse I1: N01 x dipole UV subtraction + N012 x tripole part
template <typename T>
__device__ void t_i1(const Trip<T>& t, T x01sq, T& uvsub, T& trip)
{
    const T egamma = (T)1.7810724179901979;  // exp(Euler gamma)
    const T z0 = t.z0, z1 = t.z1, z2 = t.z2;
    uvsub = 0;
    T jk = 0;
    SideSing<T> ss[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const T P = side_P(t, s), A = side_A(t, s);
        const T M2 = t.Qb2[s] + t.m2;
        const K01<T> kd = bessel_k01(DM<T>::sqrt(x01sq * M2));
        const T damp = -DM<T>::exp(-t.x2sq[s] / (x01sq * egamma));
        uvsub += P / t.x2sq[s] * damp * (A * M2 * kd.k1 * kd.k1 + t.m2 * kd.k0 * kd.k0);
        ss[s] = side_sing(t, s);
        const T X2 = side_X2(t, s);
        jk += P / t.x2sq[s] * (A * M2 * t.x3sq[s] / X2 * ss[s].k1 * ss[s].k1 + t.m2 * ss[s].k0 * ss[s].k0);
    }
    const T zj = t.zj, zk = t.zk;
    const T F = (T)0.5 * ((T)4 / (zj * zk) * f_bracket(t) * ss[0].g22 * ss[1].g22
                          - zj * z1 * z2 / (zk * zk) * t.x2jx3j * ss[1].h * ss[0].g22
                          + zk * z0 * z2 / (zj * zj) * t.x2kx3k * ss[0].h * ss[1].g22
                          - z0 * z0 * z1 * z2 / (zj * zj * zj) * t.x2jx3j * ss[0].h * ss[0].g22
                          + z1 * z1 * z0 * z2 / (zk * zk * zk) * t.x2kx3k * ss[1].h * ss[1].g22
                          + (z0 * z2) * (z0 * z2) / ((T)8 * zj * zj * zj * zj) * ss[0].h * ss[0].h
                          + (z1 * z2) * (z1 * z2) / ((T)8 * zk * zk * zk * zk) * ss[1].h * ss[1].h);
    const T c2 = ((T)2 * z0 + z2) * ((T)2 * z1 + z2) + z2 * z2;
    const T Fm = (T)0.5 * t.m2 * (-c2 * t.x20x21 * (T)2 * ss[0].g12 * ss[1].g12 / (zj * zk));
    trip = jk + F + Fm;
}

// longitudinal I1 (dis/longitudinal.py:159-214)
template <typename T>
__device__ void l_i1(const Trip<T>& t, T x01sq, T& uvsub, T& trip)
{
    const T egamma = (T)1.7810724179901979;
    const T z0 = t.z0, z1 = t.z1, z2 = t.z2;
    const T ff = (T)4 * t.Q2;
    T b[2];
    uvsub = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const T za = s == 0 ? z1 : z0, zb = s == 0 ? z0 : z1;
        const T M2 = t.Qb2[s] + t.m2;
        b[s] = bessel_k0(DM<T>::sqrt(M2) * DM<T>::sqrt(side_X2(t, s)));
        const T kd = bessel_k0(DM<T>::sqrt(M2) * DM<T>::sqrt(x01sq));
        uvsub -= za * za * ((T)2 * zb * (zb + z2) + z2 * z2) / t.x2sq[s] * DM<T>::exp(-t.x2sq[s] / x01sq / egamma) * kd * kd;
    }
    uvsub *= ff;
    trip = ff * (z1 * z1 * ((T)2 * z0 * t.zj + z2 * z2) / t.x2sq[0] * b[0] * b[0]
                 + z0 * z0 * ((T)2 * z1 * t.zk + z2 * z2) / t.x2sq[1] * b[1] * b[1]
                 - (T)2 * z0 * z1 * (z0 * ((T)1 - z0) + z1 * ((T)1 - z1)) * t.x20x21 / (t.x2sq[0] * t.x2sq[1]) * b[0] * b[1]);
}

// The G values of one auxiliary variable y: Gbar22, Gbar12, G21, G11 per side
// (G_integrand_simplified, dis/longitudinal.py:303-334, and _G_bar).
template <typename T>
struct GSet {
    T g22[2], g12[2], g21[2], g11[2];
};

// F1(z) = z K1(z) and F2(z) = z^2 K2(z) carry the A-dependence of G12 and G22 at fixed
// B and y: with z = sqrt(A B / y),
//   G12 = 4 omega/(y B) F1(z),   G22 = 8 omega/B^2 F2(z),
// so Gbar = G(lambda) - G(0) is a difference of F between z0 (lambda = 0) and z1.  When
// z1 - z0 is small that difference cancels; FP32 then integrates F' over [z0, z1] by the
// Euler-Maclaurin formula through the h^4 term, whose derivatives follow from K0, K1 at the
// two end points (d/dz z^nu K_nu = -z^nu K_{nu-1}, K0' = -K1, K1' = -K0 - K1/z):
//   dF1 = -z K0,    d2F1 = z K1 - K0,      d4F1 = z K1 - 2 K0 - K1/z
//   dF2 = -z^2 K1,  d2F2 = z^2 K0 - z K1,  d4F2 = (3 + z^2) K0 - 4 z K1
struct FDiff {
    float d1, d2;  // F1(z1) - F1(z0), F2(z1) - F2(z0)
};

__device__ __forceinline__ FDiff f_differences_em(float z0, float z1, float h, const K01<float>& a,
                                                  const K01<float>& b)
{
    const float h2 = h * h;
    const float e2 = h2 * (1.0f / 12.0f), e4 = h2 * h2 * (1.0f / 720.0f);
    FDiff o;
    {
        const float f0 = -z0 * a.k0, f1 = -z1 * b.k0;
        const float g0 = z0 * a.k1 - a.k0, g1 = z1 * b.k1 - b.k0;
        const float q0 = z0 * a.k1 - 2.0f * a.k0 - a.k1 / z0, q1 = z1 * b.k1 - 2.0f * b.k0 - b.k1 / z1;
        o.d1 = 0.5f * h * (f0 + f1) - e2 * (g1 - g0) + e4 * (q1 - q0);
    }
    {
        const float f0 = -z0 * z0 * a.k1, f1 = -z1 * z1 * b.k1;
        const float g0 = z0 * z0 * a.k0 - z0 * a.k1, g1 = z1 * z1 * b.k0 - z1 * b.k1;
        const float q0 = (3.0f + z0 * z0) * a.k0 - 4.0f * z0 * a.k1, q1 = (3.0f + z1 * z1) * b.k0 - 4.0f * z1 * b.k1;
        o.d2 = 0.5f * h * (f0 + f1) - e2 * (g1 - g0) + e4 * (q1 - q0);
    }
    return o;
}

template <typename T>
__device__ __forceinline__ void g_values_side(const Trip<T>& t, int s, T y, T& g22b, T& g12b, T& g21, T& g11)
{
    const T M2 = t.Qb2[s] + t.m2;
    const T B = y * t.x3sq[s] + t.omega[s] * t.x2sq[s];
    const T iy = (T)1 / y;
    const T delta = y * t.lam[s] * t.m2;
    const T Al = delta + M2;
    const T argl = DM<T>::sqrt(Al * B * iy);
    const T arg0 = DM<T>::sqrt(M2 * B * iy);
    const K01<T> kl = bessel_k01(argl);
    const K01<T> k0 = bessel_k01(arg0);
    const T rl = Al / B, r0 = M2 / B;
    const T sl = DM<T>::sqrt(rl), s0 = DM<T>::sqrt(r0);
    const T om = t.omega[s];
    const T sqy = DM<T>::sqrt(y);
    bool direct = true;
    if constexpr (sizeof(T) == 4) {
        // z1 - z0 = sqrt(B/y) delta / (sqrt(Al) + sqrt(M2)), free of cancellation
        const float h = DM<T>::sqrt(B * iy) * delta / (DM<T>::sqrt(Al) + DM<T>::sqrt(M2));
        if (h < 0.3f && h < 0.1f * arg0) {
            const FDiff d = f_differences_em(arg0, argl, h, k0, kl);
            g12b = 4.0f * om * iy / B * d.d1;
            g22b = 8.0f * om / (B * B) * d.d2;
            direct = false;
        }
    }
    if (direct) {
        const T k2l = kl.k0 + (T)2 * kl.k1 / argl;
        const T k20 = k0.k0 + (T)2 * k0.k1 / arg0;
        g22b = (T)8 * iy * om * (rl * k2l - r0 * k20);
        g12b = (T)4 * iy / sqy * om * (sl * kl.k1 - s0 * k0.k1);
    }
    g21 = (T)4 / sqy * sl * kl.k1;
    g11 = (T)2 * iy * kl.k0;
}

template <typename T>
__device__ __forceinline__ GSet<T> g_values(const Trip<T>& t, T y)
{
    GSet<T> g;
#pragma unroll
    for (int s = 0; s < 2; ++s) g_values_side(t, s, y, g.g22[s], g.g12[s], g.g21[s], g.g11[s]);
    return g;
}

// _IT_tripole_I2 (dis/transverse.py:565-735) over one G set
template <typename T>
__device__ T t_i2(const Trip<T>& t, const GSet<T>& G)
{
    const T z0 = t.z0, z1 = t.z1, z2 = t.z2, zj = t.zj, zk = t.zk, m2 = t.m2;
    SideSing<T> ss[2];
    T jk = 0, jkm = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        ss[s] = side_sing(t, s);
        const T M2 = t.Qb2[s] + m2;
        const T X2 = side_X2(t, s);
        jk += side_P(t, s) * side_A(t, s) * G.g22[s] * t.x3sq[s] * (T)0.125 * DM<T>::sqrt(M2 / X2) * ss[s].k1;
        jkm += side_P(t, s) * G.g12[s] * (T)0.25 * ss[s].k0;
    }
    const T F = (T)0.5 * (f_bracket(t) / ((T)4 * zj * zk) * (G.g22[1] * ss[0].g22 + G.g22[0] * ss[1].g22)
                          - zj * z1 * z2 / ((T)16 * zk * zk) * t.x2jx3j * ss[1].h * G.g22[0]
                          + zk * z0 * z2 / ((T)16 * zj * zj) * t.x2kx3k * ss[0].h * G.g22[1]
                          - z0 * z0 * z1 * z2 / ((T)16 * zj * zj * zj) * t.x2jx3j * ss[0].h * G.g22[0]
                          + z1 * z1 * z0 * z2 / ((T)16 * zk * zk * zk) * t.x2kx3k * ss[1].h * G.g22[1]);
    const T c2 = ((T)2 * z0 + z2) * ((T)2 * z1 + z2) + z2 * z2;
    const T zz2 = z2 * z2;
    const T Fm = (T)0.5 * m2
               * (-z0 * z1 * zz2 / ((T)2 * zj * zj * zj) * t.x2jx3j * G.g21[0] * ss[0].g12
                  + z0 * z1 * zz2 / ((T)2 * zk * zk * zk) * t.x2kx3k * G.g21[1] * ss[1].g12
                  - c2 * t.x20x21 / ((T)4 * zj * zk) * (G.g12[1] * ss[0].g12 + G.g12[0] * ss[1].g12)
                  - (z0 * z2) * (z0 * z2) / ((T)2 * zj * zk * zk) * t.x2jx3k * G.g21[1] * ss[0].g12
                  + (z1 * z2) * (z1 * z2) / ((T)2 * zj * zj * zk) * t.x2kx3j * G.g21[0] * ss[1].g12
                  - z0 * z1 * zz2 / (zj * zj * zj) * t.x2jx3j * G.g11[0] * ss[0].g22
                  + z0 * z1 * zz2 / (zk * zk * zk) * t.x2kx3k * G.g11[1] * ss[1].g22
                  - zj * zz2 / (zk * zk) * t.x2jx3j * G.g11[1] * ss[0].g22
                  + zk * zz2 / (zj * zj) * t.x2kx3k * G.g11[0] * ss[1].g22
                  + z0 * zz2 * z2 / ((T)4 * zj * zj * zj * zj) * ss[0].h * G.g11[0]
                  + z1 * zz2 * z2 / ((T)4 * zk * zk * zk * zk) * ss[1].h * G.g11[1]);
    return jk + m2 * jkm + F + Fm;
}

// _IT_tripole_I3 (dis/transverse.py:738-934) with G1 = G(y_t1), G2 = G(y_t2)
template <typename T>
__device__ T t_i3(const Trip<T>& t, const GSet<T>& G1, const GSet<T>& G2)
{
    const T z0 = t.z0, z1 = t.z1, z2 = t.z2, zj = t.zj, zk = t.zk, m2 = t.m2;
    T jkm = 0, jk = 0;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        jkm += side_P(t, s) * t.x2sq[s] * ((T)1 / 64) * G1.g12[s] * G2.g12[s];
        jk += side_P(t, s) * side_A(t, s) * t.x3sq[s] * t.x2sq[s] * ((T)1 / 256) * G1.g22[s] * G2.g22[s];
    }
    const T F = (T)0.5 * G1.g22[0] * G2.g22[1] / ((T)64 * zj * zk) * f_bracket(t);
    const T c2 = ((T)2 * z0 + z2) * ((T)2 * z1 + z2) + z2 * z2;
    const T zz2 = z2 * z2, z4 = zz2 * zz2;
    const T zj2 = zj * zj, zk2 = zk * zk;
    const T Fm = (T)0.5 * m2
               * (z4 / ((T)64 * zj2 * zj2) * ((T)4 * z1 * (z1 - (T)1) + (T)2) * t.x3sq[0] * G1.g21[0] * G2.g21[0]
                  + z4 / ((T)64 * zk2 * zk2) * ((T)4 * z0 * (z0 - (T)1) + (T)2) * t.x3sq[1] * G1.g21[1] * G2.g21[1]
                  - z0 * z1 * zz2 / ((T)16 * zj2 * zj) * t.x2jx3j * G1.g12[0] * G2.g21[0]
                  + z0 * z1 * zz2 / ((T)16 * zk2 * zk) * t.x2kx3k * G1.g12[1] * G2.g21[1]
                  - c2 * t.x20x21 / ((T)32 * zj * zk) * G1.g12[0] * G2.g12[1]
                  + z4 / ((T)32 * zj2 * zk2) * c2 * t.x3jx3k * G1.g21[0] * G2.g21[1]
                  + m2 * (T)0.125 * (z2 / zj) * (z2 / zj) * (z2 / zj) * (z2 / zj) * G1.g11[0] * G2.g11[0]
                  + m2 * (T)0.125 * (z2 / zk) * (z2 / zk) * (z2 / zk) * (z2 / zk) * G1.g11[1] * G2.g11[1]
                  - (z0 * z2) * (z0 * z2) / ((T)16 * zj * zk2) * t.x2jx3k * G1.g12[0] * G2.g21[1]
                  + (z1 * z2) * (z1 * z2) / ((T)16 * zk * zj2) * t.x2kx3j * G1.g12[1] * G2.g21[0]
                  - z0 * z1 * zz2 / ((T)16 * zj2 * zj) * t.x2jx3j * G1.g11[0] * G2.g22[0]
                  + z0 * z1 * zz2 / ((T)16 * zk2 * zk) * t.x2kx3k * G1.g11[1] * G2.g22[1]
                  - zj * zz2 / ((T)16 * zk2) * t.x2jx3j * G1.g11[1] * G2.g22[0]
                  + zk * zz2 / ((T)16 * zj2) * t.x2kx3k * G1.g11[0] * G2.g22[1]);
    return jk + m2 * jkm + F + Fm;
}

// longitudinal I2 / I3 (dis/longitudinal.py:217-300)
template <typename T>
__device__ T l_i2(const Trip<T>& t, const GSet<T>& G)
{
    const T z0 = t.z0, z1 = t.z1, z2 = t.z2;
    T b[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) b[s] = bessel_k0(DM<T>::sqrt(t.Qb2[s] + t.m2) * DM<T>::sqrt(side_X2(t, s)));
    return (T)4 * t.Q2
         * (z1 * z1 * ((T)2 * z0 * t.zj + z2 * z2) * (T)0.25 * G.g12[0] * b[0]
            + z0 * z0 * ((T)2 * z1 * t.zk + z2 * z2) * (T)0.25 * G.g12[1] * b[1]
            - z0 * z1 * (z0 * ((T)1 - z0) + z1 * ((T)1 - z1)) * t.x20x21 * (T)0.25
                  * (G.g12[0] * b[1] / t.x2sq[1] + G.g12[1] * b[0] / t.x2sq[0]));
}

template <typename T>
__device__ T l_i3(const Trip<T>& t, const GSet<T>& G1, const GSet<T>& G2)
{
    const T z0 = t.z0, z1 = t.z1, z2 = t.z2;
    const T zz2 = z2 * z2;
    const T a = z1 / t.zj, c = z0 / t.zk;
    return (T)4 * t.Q2
         * (z1 * z1 * ((T)2 * z0 * t.zj + zz2) * t.x2sq[0] * ((T)1 / 64) * G1.g12[0] * G2.g12[0]
            + z0 * z0 * ((T)2 * z1 * t.zk + zz2) * t.x2sq[1] * ((T)1 / 64) * G1.g12[1] * G2.g12[1]
            - z1 * z0 * (z1 * ((T)1 - z1) + z0 * ((T)1 - z0)) * t.x20x21 * ((T)1 / 32) * G1.g12[0] * G2.g12[1]
            + t.m2 * ((T)1 / 16) * zz2 * zz2
                  * (a * a * G1.g11[0] * G2.g11[0] + c * c * G1.g11[1] * G2.g11[1]
                     - (T)2 * c * a * G1.g11[0] * G2.g11[1]));
}

// FP32 form of the moment loop.  Per node y the reciprocal 1/y is shared by the two sides;
// per side the quantities that do not depend on y (M2 = Qbar^2 + m^2, its square root,
// lambda m^2, x3^2, omega x2^2) are formed once.  With q = sqrt(B/y):
//   z0 = sqrt(M2) q,  z1 = sqrt(A1) q,  z1 - z0 = q delta/(sqrt(A1)+sqrt(M2)),
// so each (node, side) needs two square roots and two reciprocals besides the Bessel pairs.
__device__ __forceinline__ K01<float> bessel_k01_rcp(float x, float& rx)
{
    rx = rcp_approx_f(x);
    return bessel_k01_from_rcp(x, rx);
}

__device__ __forceinline__ GSet<float> g_moments_f32(const Trip<float>& t, const InnerRule& rule)
{
    // The side constants of the moments (8 omega, 4 omega, 4, 2) are applied after the
    // loop, and sqrt(y) cancels between sqrt(A/B) = z sqrt(y)/B and the 1/sqrt(y) of the
    // G functions:
    //   G11 = 2 sum w/y K0(z1)             G21 = 4 sum w/B z1 K1(z1)
    //   G12 = 4 omega sum w/(y B) D12      G22 = 8 omega sum w/B E
    // with D12 = z1 K1(z1) - z0 K1(z0) (or the Euler-Maclaurin d1) and
    // E = (A1 F(z1) - M2 F(z0))/y, F(z) = K0 + 2 K1/z (or d2/B).
    float acc22[2], acc12[2], acc21[2], acc11[2];
    float M2[2], sM2[2], lm2[2], x3[2], wx2[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        acc22[s] = acc12[s] = acc21[s] = acc11[s] = 0.0f;
        M2[s] = t.Qb2[s] + t.m2;
        sM2[s] = sqrtf(M2[s]);
        lm2[s] = t.lam[s] * t.m2;
        x3[s] = t.x3sq[s];
        wx2[s] = t.omega[s] * t.x2sq[s];
    }
    for (int i = 0; i < rule.n; ++i) {
        const float y = (float)rule.y[i];
        const float w = (float)rule.w[i];
        const float iy = rcp_approx_f(y);
        const float wiy = w * iy;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const float B = fmaf(y, x3[s], wx2[s]);
            const float iB = rcp_approx_f(B);
            const float q = sqrtf(B * iy);
            const float delta = y * lm2[s];
            const float Al = delta + M2[s];
            const float sAl = sqrtf(Al);
            const float z1 = sAl * q, z0 = sM2[s] * q;
            float r1, r0;
            const K01<float> kl = bessel_k01_rcp(z1, r1);
            const K01<float> k0 = bessel_k01_rcp(z0, r0);
            const float h = q * delta * rcp_approx_f(sAl + sM2[s]);
            const float z1k1 = z1 * kl.k1;
            float d12, e22;
            if (h < 0.3f && h < 0.1f * z0) {
                // Euler-Maclaurin integral of dF/dz over [z0, z1] (see f_differences_em)
                const float h2 = h * h;
                const float e2 = h2 * (1.0f / 12.0f), e4 = h2 * h2 * (1.0f / 720.0f);
                const float d1 = 0.5f * h * (-z0 * k0.k0 - z1 * kl.k0) -
                                 e2 * ((z1k1 - kl.k0) - (z0 * k0.k1 - k0.k0)) +
                                 e4 * ((z1k1 - 2.0f * kl.k0 - kl.k1 * r1) - (z0 * k0.k1 - 2.0f * k0.k0 - k0.k1 * r0));
                const float d2 = 0.5f * h * (-z0 * z0 * k0.k1 - z1 * z1k1) -
                                 e2 * ((z1 * z1 * kl.k0 - z1k1) - (z0 * z0 * k0.k0 - z0 * k0.k1)) +
                                 e4 * (((3.0f + z1 * z1) * kl.k0 - 4.0f * z1k1) -
                                       ((3.0f + z0 * z0) * k0.k0 - 4.0f * z0 * k0.k1));
                d12 = d1;
                e22 = iB * d2;
            } else {
                d12 = z1k1 - z0 * k0.k1;
                e22 = iy * (Al * fmaf(2.0f * kl.k1, r1, kl.k0) - M2[s] * fmaf(2.0f * k0.k1, r0, k0.k0));
            }
            const float wiB = w * iB;
            acc22[s] = fmaf(wiB, e22, acc22[s]);
            acc12[s] = fmaf(wiy * iB, d12, acc12[s]);
            acc21[s] = fmaf(wiB, z1k1, acc21[s]);
            acc11[s] = fmaf(wiy, kl.k0, acc11[s]);
        }
    }
    GSet<float> m;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        m.g22[s] = 8.0f * t.omega[s] * acc22[s];
        m.g12[s] = 4.0f * t.omega[s] * acc12[s];
        m.g21[s] = 4.0f * acc21[s];
        m.g11[s] = 2.0f * acc11[s];
    }
    return m;
}

template <typename T>
__device__ __forceinline__ GSet<T> g_moments(const Trip<T>& t, const InnerRule& rule)
{
    if constexpr (sizeof(T) == 4) return g_moments_f32(t, rule);
    GSet<T> m;
#pragma unroll
    for (int s = 0; s < 2; ++s) m.g22[s] = m.g12[s] = m.g21[s] = m.g11[s] = (T)0;
    for (int i = 0; i < rule.n; ++i) {
        const GSet<T> g = g_values(t, (T)rule.y[i]);
        const T w = (T)rule.w[i];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            m.g22[s] = fma(w, g.g22[s], m.g22[s]);
            m.g12[s] = fma(w, g.g12[s], m.g12[s]);
            m.g21[s] = fma(w, g.g21[s], m.g21[s]);
            m.g11[s] = fma(w, g.g11[s], m.g11[s]);
        }
    }
    return m;
}

// integrand_qgunsub_massive (dis/observables.py:175-250) and the nested forms
// (integrand_qg_nested_massive, :253-331)
template <typename T, int TERM>
__device__ T qg_term(const DisArgs<T>& a, const double* x, const InnerRule& rule)
{
    const double z2min = a.z2min;
    if (z2min > 1.0) return (T)0;
    const double z1 = (1.0 - z2min) * x[0];
    const double z2 = (1.0 - z1 - z2min) * x[1] + z2min;
    const double x01 = a.maxr * x[2];
    const double x02 = a.maxr * x[3];
    const double phi = 2.0 * kPi * x[4];
    const double x01sq = x01 * x01, x02sq = x02 * x02;
    double x21sq = x01sq + x02sq - 2.0 * x01 * x02 * ::cos(phi);
    x21sq = x21sq > 0.0 ? x21sq : 0.0;
    const double x21 = ::sqrt(x21sq);
    const double jac = (1.0 - z2min) * (1.0 - z1 - z2min) * x01 * x02 * a.maxr * a.maxr * 2.0 * kPi;
    const double Y = ::log(a.W2 * z2 / kQ0sqr);
    if (!(Y >= 0.0)) return (T)0;
    T N01, N02, N21;
    amplitudes3(a, x01, x02, x21, Y, N01, N02, N21);
    const T S01 = (T)1 - N01;
    const T S02 = (T)1 - N02;
    const T S12 = (T)1 - N21;
    const T N012 = a.finite_nc ? (T)1 - (T)(kNc / (2.0 * kCF)) * (S02 * S12 - S01 / (T)(kNc * kNc))
                               : (T)1 - S02 * S12;
    const double ra = a.parent_coupling ? x01 : fmin(x01, fmin(x02, x21));
    const T af = alpha_bar(a, (T)ra);
    const Trip<T> t = make_trip<T>(a.Q2, a.mf, z1, z2, x01sq, x02sq, x21sq);
    T v;
    if constexpr (TERM == kTermI1) {
        T uvsub, trip;
        if (a.transverse)
            t_i1(t, (T)x01sq, uvsub, trip);
        else
            l_i1(t, (T)x01sq, uvsub, trip);
        v = ((T)1 - S01) * uvsub + N012 * trip;
    } else if constexpr (TERM == kTermI2 || TERM == kTermI2N) {
        GSet<T> G;
        if constexpr (TERM == kTermI2)
            G = g_values(t, (T)x[5]);
        else
            G = g_moments(t, rule);
        v = N012 * (a.transverse ? t_i2(t, G) : l_i2(t, G));
    } else {
        if constexpr (TERM == kTermI3) {
            const GSet<T> G1 = g_values(t, (T)x[5]);
            const GSet<T> G2 = g_values(t, (T)x[6]);
            v = N012 * (a.transverse ? t_i3(t, G1, G2) : l_i3(t, G1, G2));
        } else {
            const GSet<T> G = g_moments(t, rule);
            v = N012 * (a.transverse ? t_i3(t, G, G) : l_i3(t, G, G));
        }
    }
    const T out = v * (T)(jac / z2) * af;
    return DM<T>::finite(out) ? out : (T)0;
}

// I1, and I2 and I3 with the inner rule, at one point: the map, the amplitudes, the
// coupling and the tripole geometry are shared, and I2 and I3 use one moment set (the
// combined evaluation of the fixed-Sobol path, dis/fixed_sobol.py:273-368).
template <typename T>
__device__ void qg_triple(const DisArgs<T>& a, const double* x, const InnerRule& rule, T out[3])
{
    out[0] = out[1] = out[2] = (T)0;
    const double z2min = a.z2min;
    if (z2min > 1.0) return;
    const double z1 = (1.0 - z2min) * x[0];
    const double z2 = (1.0 - z1 - z2min) * x[1] + z2min;
    const double x01 = a.maxr * x[2];
    const double x02 = a.maxr * x[3];
    const double phi = 2.0 * kPi * x[4];
    const double x01sq = x01 * x01, x02sq = x02 * x02;
    double x21sq = x01sq + x02sq - 2.0 * x01 * x02 * ::cos(phi);
    x21sq = x21sq > 0.0 ? x21sq : 0.0;
    const double x21 = ::sqrt(x21sq);
    const double jac = (1.0 - z2min) * (1.0 - z1 - z2min) * x01 * x02 * a.maxr * a.maxr * 2.0 * kPi;
    const double Y = ::log(a.W2 * z2 / kQ0sqr);
    if (!(Y >= 0.0)) return;
    T N01, N02, N21;
    amplitudes3(a, x01, x02, x21, Y, N01, N02, N21);
    const T S01 = (T)1 - N01;
    const T S02 = (T)1 - N02;
    const T S12 = (T)1 - N21;
    const T N012 = a.finite_nc ? (T)1 - (T)(kNc / (2.0 * kCF)) * (S02 * S12 - S01 / (T)(kNc * kNc))
                               : (T)1 - S02 * S12;
    const double ra = a.parent_coupling ? x01 : fmin(x01, fmin(x02, x21));
    const T scale = alpha_bar(a, (T)ra) * (T)(jac / z2);
    const Trip<T> t = make_trip<T>(a.Q2, a.mf, z1, z2, x01sq, x02sq, x21sq);
    T uvsub, trip;
    if (a.transverse)
        t_i1(t, (T)x01sq, uvsub, trip);
    else
        l_i1(t, (T)x01sq, uvsub, trip);
    const GSet<T> G = g_moments(t, rule);
    const T i1 = (((T)1 - S01) * uvsub + N012 * trip) * scale;
    const T i2 = N012 * (a.transverse ? t_i2(t, G) : l_i2(t, G)) * scale;
    const T i3 = N012 * (a.transverse ? t_i3(t, G, G) : l_i3(t, G, G)) * scale;
    out[0] = DM<T>::finite(i1) ? i1 : (T)0;
    out[1] = DM<T>::finite(i2) ? i2 : (T)0;
    out[2] = DM<T>::finite(i3) ? i3 : (T)0;
}

template <typename T, int TERM>
__device__ __forceinline__ T term_value(const DisArgs<T>& a, const double* x, const InnerRule& rule)
{
    if constexpr (TERM == kTermLO)
        return lo_term(a, x);
    else if constexpr (TERM == kTermDip0)
        return dip_term<T, 0>(a, x);
    else if constexpr (TERM == kTermDip1)
        return dip_term<T, 1>(a, x);
    else if constexpr (TERM == kTermDip2)
        return dip_term<T, 2>(a, x);
    else
        return qg_term<T, TERM>(a, x, rule);
}

}  // namespace dis
}  // namespace nlo
