// BK-table dipole amplitude N(r, Y) on the device (dipole/amplitude.py:48-252).
//
// A prepared table is one device buffer of doubles (nlo_dis_table_doubles):
//   header[16] | r[nr] | Y[ny] | N[ny*nr] | window[nr-1][20] | global[nr-1][4]
//   | local[ny][nr-1][4]
// window[i] describes the local spline used for r in [r_i, r_{i+1}): the reference takes
// the 7 table points starting at max(i-3, 0) (the last 9 points when i+3 > nr-1), fills
// them with N linearly interpolated in Y, fits a natural cubic spline in r and evaluates
// it on interval i - start (dipole/amplitude.py:215-252).  The spline's second
// derivatives are linear in the 7/9 values, so the prepare kernel stores, per interval,
// the window start (slot 0), the point count (slot 1) and the two rows of that linear
// map that the interval needs (slots 2..19: M_j and M_{j+1} as weights over 9 values).
// Because the whole spline is linear in the window values, the spline of the
// Y-interpolated values is the same interpolation of the splines of the two stored rows:
// local[k][i] holds the power-form coefficients (a, b, c, d) of row k's window spline on
// interval i, and an evaluation blends two of them and runs one cubic.
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
    kHdrY0 = 12,      // Y[0] (table rows, x0 shift included)
    kHdrInvDY = 13,   // (ny - 1) / (Y[ny-1] - Y[0]), 0 for one row
};

struct TableView {
    const double* hdr;
    const double* r;
    const double* Y;
    const double* N;
    const double* window;
    const double* global;
    const double* local;
    int nr, ny;
};

__host__ __device__ inline size_t table_doubles(int nr, int ny)
{
    return (size_t)kTableHeader + nr + ny + (size_t)ny * nr + (size_t)(nr - 1) * kWindowStride + (size_t)(nr - 1) * 4 +
           (size_t)ny * (nr - 1) * 4;
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
    v.local = v.global + (size_t)(nr - 1) * 4;
    v.nr = nr;
    v.ny = ny;
    return v;
}

// Largest k in [0, n) with x_k <= v, or -1 (searchsorted(x, v, right) - 1), from a guess
// that a uniform grid in the lookup variable would give.  The guess is corrected by a few
// steps against the stored knots and verified; a grid far from uniform falls back to a
// binary search, so the result never depends on the guess.
__device__ __forceinline__ int knot_index(const double* __restrict__ x, int n, double v, double guess)
{
    int k = guess >= -1.0 && guess < (double)n ? (int)floor(guess) : (guess >= (double)n ? n - 1 : -1);
    for (int step = 0; step < 4 && k >= 0 && !(x[k] <= v); ++step) --k;
    for (int step = 0; step < 4 && k + 1 < n && x[k + 1] <= v; ++step) ++k;
    if ((k < 0 || x[k] <= v) && (k + 1 >= n || !(x[k + 1] <= v))) return k;
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (x[mid] <= v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo - 1;
}

// interval i in [0, nr-2] with r_i <= r < r_{i+1} (clamped); the guess takes the log of r
// in FP32, which the correction makes exact
__device__ __forceinline__ int table_r_interval(const TableView& t, double r)
{
    const double guess = ((double)__logf((float)r) - t.hdr[kHdrLogR0]) * t.hdr[kHdrInvDlogR];
    const int i = knot_index(t.r, t.nr, r, guess);
    return i < 0 ? 0 : (i > t.nr - 2 ? t.nr - 2 : i);
}

// The rapidity side of a lookup, shared by every amplitude at one Y: the two table rows,
// the interpolation fraction and whether the initialised global spline applies.
struct TableRow {
    double Y, frac;
    int lo, hi;
    bool global;
};

__device__ __forceinline__ bool table_initialized_at(const TableView& t, double Y)
{
    if (t.hdr[kHdrInitialized] == 0.0) return false;
    const double iy = t.hdr[kHdrInitY];
    if (::fabs(Y) < 0.001 && ::fabs(iy) < 0.001) return true;
    const double den = Y < iy ? Y : iy;
    const double safe = den != 0.0 ? den : 1.0;
    return iy >= 0.0 && ::fabs(Y - iy) / safe < 0.001;
}

// dipole_amplitude's rapidity handling (dipole/amplitude.py:135-170, 215-230): Y below
// the first row frozen to it, rows yind = searchsorted(Y, right) - 1 (0 below the table)
// and yind + 1 (the last row above it), linear fraction between them.
__device__ __forceinline__ TableRow table_row(const TableView& t, double Y)
{
    const double ymin = t.hdr[kHdrYmin], ymax = t.hdr[kHdrYmax];
    if (Y >= 0.0 && Y < ymin) Y = ymin;
    if (Y > ymax) Y = ymax;  // the host rejects requests that reach beyond the table
    TableRow row;
    row.Y = Y;
    int yind = knot_index(t.Y, t.ny, Y, (Y - t.hdr[kHdrY0]) * t.hdr[kHdrInvDY]);
    yind = yind < 0 ? 0 : yind;
    const int yind2 = yind + 1 < t.ny ? yind + 1 : t.ny - 1;
    row.lo = yind;
    row.hi = yind2;
    row.frac = yind2 != yind ? (Y - t.Y[yind]) / (t.Y[yind2] - t.Y[yind]) : 0.0;
    row.global = table_initialized_at(t, Y);
    return row;
}

// The local spline (dipole/amplitude.py:215-252) from the two rows' coefficients.
__device__ __forceinline__ double table_local(const TableView& t, const TableRow& row, double r, int rind)
{
    const double* lo = t.local + ((size_t)row.lo * (t.nr - 1) + rind) * 4;
    const double* hi = t.local + ((size_t)row.hi * (t.nr - 1) + rind) * 4;
    const double f = row.frac;
    const double a = fma(f, hi[0] - lo[0], lo[0]);
    const double b = fma(f, hi[1] - lo[1], lo[1]);
    const double c = fma(f, hi[2] - lo[2], lo[2]);
    const double d = fma(f, hi[3] - lo[3], lo[3]);
    const double dx = r - t.r[rind];
    return a + dx * (b + dx * (c + dx * d));
}

// LINEAR_LINEAR (dipole/amplitude.py:188-212), the reference's expression order: the
// last Y row interpolates in r only, and r on (or past) the last knot gives 1.
__device__ __forceinline__ double table_bilinear(const TableView& t, const TableRow& row, double r, int rind)
{
    if (r >= t.r[t.nr - 1]) return 1.0;
    const double r1 = t.r[rind], r2 = t.r[rind + 1];
    const double* lo = t.N + (size_t)row.lo * t.nr + rind;
    const double N11 = lo[0], N12 = lo[1];
    if (row.hi == row.lo) return N11 + (r - r1) / (r2 - r1) * (N12 - N11);
    const double* hi = t.N + (size_t)row.hi * t.nr + rind;
    const double N21 = hi[0], N22 = hi[1];
    const double Y = row.Y, Y1 = t.Y[row.lo], Y2 = t.Y[row.hi];
    return (N11 * (r2 - r) * (Y2 - Y) + N12 * (r - r1) * (Y2 - Y) + N21 * (r2 - r) * (Y - Y1) +
            N22 * (r - r1) * (Y - Y1)) /
           ((r2 - r1) * (Y2 - Y1));
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

// dipole_amplitude (dipole/amplitude.py:135-170) at a prepared rapidity: r clamped into
// the table, the initialised global spline when Y matches, the local spline (or the
// bilinear rule) else; the result clamped to [0, 1].
__device__ __forceinline__ double table_amplitude_at(const TableView& t, const TableRow& row, double r)
{
    const double rmin = t.hdr[kHdrRmin], rmax = t.hdr[kHdrRmax];
    if (r < rmin) r = rmin * 1.000001;
    if (r > rmax) r = rmax * 0.999999;
    const int rind = table_r_interval(t, r);
    const double v = row.global                 ? table_global(t, r, rind)
                     : t.hdr[kHdrInterp] != 0.0 ? table_bilinear(t, row, r, rind)
                                                : table_local(t, row, r, rind);
    return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
}

__device__ __forceinline__ double table_amplitude(const TableView& t, double r, double Y)
{
    return table_amplitude_at(t, table_row(t, Y), r);
}

}  // namespace dis
}  // namespace nlo
