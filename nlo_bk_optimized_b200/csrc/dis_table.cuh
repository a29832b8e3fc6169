// BK-table dipole amplitude N(r, Y) on the device (dipole/amplitude.py:48-252).
//
// A prepared table is one device buffer of doubles (nlo_dis_table_doubles):
//   header[16] | r[nr] | Y[ny] | N[ny*nr] | window[nr-1][20] | global[nr-1][4]
// window[i] describes the local spline used for r in [r_i, r_{i+1}): the reference takes
// the 7 table points starting at max(i-3, 0) (the last 9 points when i+3 > nr-1), fills
// them with N linearly interpolated in Y, fits a natural cubic spline in r and evaluates
// it on interval i - start (dipole/amplitude.py:215-252).  The spline's second
// derivatives are linear in the 7/9 values, so the prepare kernel stores, per interval,
// the window start (slot 0), the point count (slot 1) and the two rows of that linear
// map that the interval needs (slots 2..19: M_j and M_{j+1} as weights over 9 values).
// Evaluation is then 9 Y-interpolated loads, two dot products and one cubic.
// global[] holds the natural spline of the table at one fixed rapidity that
// initialize_interpolation builds (dipole/amplitude.py:105-133, 177-184).
// Header slot kHdrInterp selects the reference's LINEAR_LINEAR mode instead of the local
// spline (1; dipole/amplitude.py:188-212): bilinear in (r, Y) on the stored rows.
#pragma once

#include <cuda_runtime.h>

namespace nlo {
namespace dis {

constexpr int kTableHeader = 16;
constexpr int kWindowStride = 20;
constexpr int kWindowMax = 9;

// header slots
enum TableSlot {
    kHdrNr = 0,
    kHdrNy = 1,
    kHdrInitialized = 2,
    kHdrInitY = 3,
    kHdrMaxrInterp = 4,
    kHdrRmin = 5,
    kHdrRmax = 6,
    kHdrYmin = 7,
    kHdrYmax = 8,
    kHdrLogR0 = 9,
    kHdrInvDlogR = 10,
    kHdrInterp = 11,  // 0: SPLINE_LINEAR, 1: LINEAR_LINEAR
};

struct TableView {
    const double* hdr;
    const double* r;
    const double* Y;
    const double* N;
    const double* window;
    const double* global;
    int nr, ny;
};

__host__ __device__ inline size_t table_doubles(int nr, int ny)
{
    return (size_t)kTableHeader + nr + ny + (size_t)ny * nr + (size_t)(nr - 1) * kWindowStride + (size_t)(nr - 1) * 4;
}

__host__ __device__ inline TableView table_view(const double* base, int nr, int ny)
{
    TableView v;
    v.hdr = base;
    v.r = base + kTableHeader;
    v.Y = v.r + nr;
    v.N = v.Y + ny;
    v.window = v.N + (size_t)ny * nr;
    v.global = v.window + (size_t)(nr - 1) * kWindowStride;
    v.nr = nr;
    v.ny = ny;
    return v;
}

// largest i in [0, nr-2] with r_i <= r (searchsorted(right) - 1, clamped), from a
// log-grid guess corrected against the stored knots
__device__ __forceinline__ int table_r_interval(const TableView& t, double r)
{
    int i = (int)floor((::log(r) - t.hdr[kHdrLogR0]) * t.hdr[kHdrInvDlogR]);
    i = i < 0 ? 0 : (i > t.nr - 2 ? t.nr - 2 : i);
    for (int guard = 0; guard < 8 && i > 0 && r < t.r[i]; ++guard) --i;
    for (int guard = 0; guard < 8 && i < t.nr - 2 && r >= t.r[i + 1]; ++guard) ++i;
    return i;
}

__device__ __forceinline__ int table_y_index(const TableView& t, double Y)
{
    int lo = 0, hi = t.ny;  // first index with Y_k > Y, minus one
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (t.Y[mid] <= Y)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo - 1;
}

__device__ __forceinline__ double table_local(const TableView& t, double r, double Y, int rind)
{
    int yind = table_y_index(t, Y);
    yind = yind < 0 ? 0 : yind;
    const int yind2 = yind + 1 < t.ny ? yind + 1 : t.ny - 1;
    const double frac = yind2 != yind ? (Y - t.Y[yind]) / (t.Y[yind2] - t.Y[yind]) : 0.0;
    const double* w = t.window + (size_t)rind * kWindowStride;
    const int start = (int)w[0];
    const int points = (int)w[1];
    const int j = rind - start;
    const double* lo_row = t.N + (size_t)yind * t.nr + start;
    const double* hi_row = t.N + (size_t)yind2 * t.nr + start;
    double mj = 0.0, mj1 = 0.0, vj = 0.0, vj1 = 0.0;
#pragma unroll
    for (int k = 0; k < kWindowMax; ++k) {
        if (k < points) {
            const double lo = lo_row[k];
            const double v = lo + frac * (hi_row[k] - lo);
            mj = fma(w[2 + k], v, mj);
            mj1 = fma(w[2 + kWindowMax + k], v, mj1);
            if (k == j) vj = v;
            if (k == j + 1) vj1 = v;
        }
    }
    const double x0 = t.r[rind];
    const double h = t.r[rind + 1] - x0;
    const double b = (vj1 - vj) / h - h * (2.0 * mj + mj1) / 6.0;
    const double c = mj / 2.0;
    const double d = (mj1 - mj) / (6.0 * h);
    const double dx = r - x0;
    return vj + dx * (b + dx * (c + dx * d));
}

// LINEAR_LINEAR (dipole/amplitude.py:188-212), the reference's expression order: the
// last Y row interpolates in r only, and r on (or past) the last knot gives 1.
__device__ __forceinline__ double table_bilinear(const TableView& t, double r, double Y, int rind)
{
    if (r >= t.r[t.nr - 1]) return 1.0;
    int yind = table_y_index(t, Y);
    yind = yind < 0 ? 0 : yind;
    const int yind2 = yind + 1 < t.ny ? yind + 1 : t.ny - 1;
    const double r1 = t.r[rind], r2 = t.r[rind + 1];
    const double* lo = t.N + (size_t)yind * t.nr + rind;
    const double N11 = lo[0], N12 = lo[1];
    if (yind2 == yind) return N11 + (r - r1) / (r2 - r1) * (N12 - N11);
    const double* hi = t.N + (size_t)yind2 * t.nr + rind;
    const double N21 = hi[0], N22 = hi[1];
    const double Y1 = t.Y[yind], Y2 = t.Y[yind2];
    return (N11 * (r2 - r) * (Y2 - Y) + N12 * (r - r1) * (Y2 - Y) + N21 * (r2 - r) * (Y - Y1) +
            N22 * (r - r1) * (Y - Y1)) /
           ((r2 - r1) * (Y2 - Y1));
}

__device__ __forceinline__ bool table_initialized_at(const TableView& t, double Y)
{
    if (t.hdr[kHdrInitialized] == 0.0) return false;
    const double iy = t.hdr[kHdrInitY];
    if (::fabs(Y) < 0.001 && ::fabs(iy) < 0.001) return true;
    const double den = Y < iy ? Y : iy;
    const double safe = den != 0.0 ? den : 1.0;
    return iy >= 0.0 && ::fabs(Y - iy) / safe < 0.001;
}

__device__ __forceinline__ double table_global(const TableView& t, double r, int rind)
{
    const double* g = t.global + (size_t)rind * 4;
    const double dx = r - t.r[rind];
    double v = g[0] + dx * (g[1] + dx * (g[2] + dx * g[3]));
    const double maxr = t.hdr[kHdrMaxrInterp];
    if (maxr > 0.0 && r >= maxr) v = 1.0;
    return v;
}

// dipole_amplitude (dipole/amplitude.py:135-170): r clamped into the table, Y below the
// first row frozen to it, initialised global spline when Y matches, local spline else;
// the result clamped to [0, 1].
__device__ __forceinline__ double table_amplitude(const TableView& t, double r, double Y)
{
    const double rmin = t.hdr[kHdrRmin], rmax = t.hdr[kHdrRmax];
    if (r < rmin) r = rmin * 1.000001;
    if (r > rmax) r = rmax * 0.999999;
    const double ymin = t.hdr[kHdrYmin], ymax = t.hdr[kHdrYmax];
    if (Y >= 0.0 && Y < ymin) Y = ymin;
    if (Y > ymax) Y = ymax;  // the host rejects requests that reach beyond the table
    const int rind = table_r_interval(t, r);
    const double v = table_initialized_at(t, Y)       ? table_global(t, r, rind)
                     : t.hdr[kHdrInterp] != 0.0 ? table_bilinear(t, r, Y, rind)
                                                : table_local(t, r, Y, rind);
    return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
}

}  // namespace dis
}  // namespace nlo
