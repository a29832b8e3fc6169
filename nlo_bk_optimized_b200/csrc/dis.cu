// NLO DIS kernels (sm_100a): BK-table preparation, pointwise integrands, the tensor
// Gauss-Legendre rule of the 2D terms, and the device Vegas iteration.
//
// Vegas (numerics/integration.py:120-589, 804-866) runs entirely on the device: one
// iteration kernel per round maps scrambled Sobol points through the current grid,
// evaluates the integrand, and leaves per-CTA partial sums of w, w^2 and the |w| / count
// histograms; one finalize CTA per integral reduces the partials in a fixed order,
// re-bins the grid and updates the inverse-variance-weighted estimate and the
// convergence flag.  A converged integral makes the remaining rounds no-ops, so the host
// enqueues all rounds without synchronising.  Many integrals (jobs) of one term run in
// the same launches (grid.y = job).  Every reduction has a fixed order, so results are
// bit-reproducible run to run.
#include <cuda_runtime.h>

#include "dis_internal.h"
#include "dis_terms.cuh"
#include "sobol.cuh"
#include "vegas_common.cuh"

namespace nlo {
namespace dis {

// ===========================================================================
// Table preparation (dipole/amplitude.py:48-83, 215-252)

__global__ void table_prepare_kernel(const double* __restrict__ r, const double* __restrict__ y,
                                     const double* __restrict__ N, int nr, int ny, double y0, int interp,
                                     double* table)
{
    const TableView v = table_view(table, nr, ny);
    double* hdr = table;
    double* tr = table + kTableHeader;
    double* tY = tr + nr;
    double* tN = tY + ny;
    double* win = tN + (size_t)ny * nr;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    for (int i = tid; i < nr; i += stride) tr[i] = r[i];
    for (int i = tid; i < ny; i += stride) tY[i] = y[i] + y0;
    for (size_t i = tid; i < (size_t)ny * nr; i += stride) tN[i] = N[i];
    if (tid == 0) {
        for (int k = 0; k < kTableHeader; ++k) hdr[k] = 0.0;
        hdr[kHdrNr] = nr;
        hdr[kHdrNy] = ny;
        hdr[kHdrInitialized] = 0.0;
        hdr[kHdrInitY] = -1.0;
        hdr[kHdrMaxrInterp] = -1.0;
        hdr[kHdrRmin] = r[0];
        hdr[kHdrRmax] = r[nr - 1];
        hdr[kHdrYmin] = y[0] + y0;
        hdr[kHdrYmax] = y[ny - 1] + y0;
        hdr[kHdrLogR0] = ::log(r[0]);
        hdr[kHdrInvDlogR] = (nr - 1) / (::log(r[nr - 1]) - ::log(r[0]));
        hdr[kHdrInterp] = interp;
        hdr[kHdrY0] = y[0] + y0;
        hdr[kHdrInvDY] = ny > 1 ? (ny - 1) / ((y[ny - 1] + y0) - (y[0] + y0)) : 0.0;
    }
    // window weights: second derivatives of the natural spline through the 7/9 window
    // points as linear maps of the window values (one Thomas solve per unit vector)
    for (int i = tid; i < nr - 1; i += stride) {
        const bool upper = i + 3 > nr - 1;
        const int points = upper ? 9 : 7;
        int start = upper ? nr - 9 : i - 3;
        start = start < 0 ? 0 : start;
        const int j = i - start;
        double h[kWindowMax - 1];
        for (int k = 0; k < points - 1; ++k) h[k] = r[start + k + 1] - r[start + k];
        double* w = win + (size_t)i * kWindowStride;
        w[0] = start;
        w[1] = points;
        for (int k = 0; k < 2 * kWindowMax; ++k) w[2 + k] = 0.0;
        const int m = points - 2;  // interior unknowns
        for (int unit = 0; unit < points; ++unit) {
            double c[kWindowMax], d[kWindowMax];
            for (int q = 0; q < m; ++q) {
                // rhs_q = 6 ((e_{q+2} - e_{q+1})/h_{q+1} - (e_{q+1} - e_q)/h_q)
                const double e0 = unit == q ? 1.0 : 0.0;
                const double e1 = unit == q + 1 ? 1.0 : 0.0;
                const double e2 = unit == q + 2 ? 1.0 : 0.0;
                const double rhs = 6.0 * ((e2 - e1) / h[q + 1] - (e1 - e0) / h[q]);
                const double diag = 2.0 * (h[q] + h[q + 1]);
                if (q == 0) {
                    c[q] = m > 1 ? h[1] / diag : 0.0;
                    d[q] = rhs / diag;
                } else {
                    const double den = diag - h[q] * c[q - 1];
                    c[q] = q < m - 1 ? h[q + 1] / den : 0.0;
                    d[q] = (rhs - h[q] * d[q - 1]) / den;
                }
            }
            double M[kWindowMax];
            M[0] = 0.0;
            M[points - 1] = 0.0;
            double next = d[m - 1];
            M[m] = next;
            for (int q = m - 2; q >= 0; --q) {
                next = d[q] - c[q] * next;
                M[q + 1] = next;
            }
            w[2 + unit] = M[j];
            w[2 + kWindowMax + unit] = M[j + 1];
        }
    }
    (void)v;
}

// Per-row coefficients of the local splines: for table row k and r interval i, the
// window spline through row k's values (second derivatives from the window weights),
// in the power form a + b dx + c dx^2 + d dx^3 on [r_i, r_{i+1}).
__global__ void table_local_kernel(double* table, int nr, int ny)
{
    const TableView v = table_view(table, nr, ny);
    double* local = table + (v.local - table);
    const int64_t total = (int64_t)ny * (nr - 1);
    for (int64_t item = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; item < total;
         item += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(item / (nr - 1));
        const int i = (int)(item - (int64_t)k * (nr - 1));
        const double* w = v.window + (size_t)i * kWindowStride;
        const int start = (int)w[0];
        const int points = (int)w[1];
        const int j = i - start;
        const double* vals = v.N + (size_t)k * nr + start;
        double mj = 0.0, mj1 = 0.0;
        for (int q = 0; q < points; ++q) {
            mj = fma(w[2 + q], vals[q], mj);
            mj1 = fma(w[2 + kWindowMax + q], vals[q], mj1);
        }
        const double vj = vals[j], vj1 = vals[j + 1];
        const double h = v.r[i + 1] - v.r[i];
        double* out = local + (size_t)item * 4;
        out[0] = vj;
        out[1] = (vj1 - vj) / h - h * (2.0 * mj + mj1) / 6.0;
        out[2] = mj / 2.0;
        out[3] = (mj1 - mj) / (6.0 * h);
    }
}

// initialize_interpolation (dipole/amplitude.py:105-133) and _find_maxr_interpolate
// (:254-272): one CTA.  Threads evaluate the local amplitude at the knots (the end knots
// nudged inwards by 1e-4), thread 0 fits the natural spline in r and runs the search.
__global__ void table_initialize_kernel(double* table, int nr, int ny, double Y)
{
    extern __shared__ double smem[];
    double* vals = smem;        // [nr]
    double* cc = smem + nr;     // [nr]
    double* dd = smem + 2 * nr; // [nr]
    TableView v = table_view(table, nr, ny);
    double* hdr = table;
    if (threadIdx.x == 0) {
        hdr[kHdrInitialized] = 0.0;
        hdr[kHdrInitY] = -1.0;
        hdr[kHdrMaxrInterp] = -1.0;
    }
    __syncthreads();
    double Yv = Y;
    if (Yv >= 0.0 && Yv <= hdr[kHdrYmin]) Yv = hdr[kHdrYmin];
    for (int k = threadIdx.x; k < nr; k += blockDim.x) {
        double rr = v.r[k];
        if (k == 0) rr *= 1.0001;
        if (k == nr - 1) rr *= 0.9999;
        vals[k] = table_amplitude(v, rr, Yv);
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    // natural spline through (r_k, vals_k): interior second derivatives by Thomas
    double* g = table + (v.global - table);
    const int m = nr - 2;
    for (int q = 0; q < m; ++q) {
        const double h0 = v.r[q + 1] - v.r[q], h1 = v.r[q + 2] - v.r[q + 1];
        const double rhs = 6.0 * ((vals[q + 2] - vals[q + 1]) / h1 - (vals[q + 1] - vals[q]) / h0);
        const double diag = 2.0 * (h0 + h1);
        if (q == 0) {
            cc[q] = m > 1 ? h1 / diag : 0.0;
            dd[q] = rhs / diag;
        } else {
            const double den = diag - h0 * cc[q - 1];
            cc[q] = q < m - 1 ? h1 / den : 0.0;
            dd[q] = (rhs - h0 * dd[q - 1]) / den;
        }
    }
    // back substitution into dd (dd[q] = M_{q+1}); then the power-form coefficients
    for (int q = m - 2; q >= 0; --q) dd[q] = dd[q] - cc[q] * dd[q + 1];
    for (int k = 0; k < nr - 1; ++k) {
        const double mk = k == 0 ? 0.0 : dd[k - 1];
        const double mk1 = k + 1 == nr - 1 ? 0.0 : dd[k];
        const double h = v.r[k + 1] - v.r[k];
        g[4 * k + 0] = vals[k];
        g[4 * k + 1] = (vals[k + 1] - vals[k]) / h - h * (2.0 * mk + mk1) / 6.0;
        g[4 * k + 2] = mk / 2.0;
        g[4 * k + 3] = (mk1 - mk) / (6.0 * h);
    }
    hdr[kHdrInitY] = Yv;
    hdr[kHdrInitialized] = 1.0;
    __threadfence_block();
    double step = 2.0, previous = 0.1, rr = 0.01;
    double found = -1.0;
    for (int it = 0; it < 41; ++it) {
        if (rr > hdr[kHdrRmax]) break;
        const double val = table_amplitude(v, rr, Yv);
        if (val >= 0.99999) {
            if (step < 1e-2) {
                found = rr;
                break;
            }
            step /= 1.5;
            rr = previous;
        }
        previous = rr;
        rr += step;
    }
    hdr[kHdrMaxrInterp] = found;
}

// ===========================================================================
// Pointwise integrands (the reference's dis_*_integrand operators)

template <typename T, int TERM>
__global__ void points_kernel(const DisArgs<T> args, InnerRule rule, const double* __restrict__ x, int64_t n,
                              double* __restrict__ out)
{
    constexpr int D = term_dims(TERM);
    __shared__ __align__(16) unsigned char raw[sizeof(DisArgs<T>)];
    DisArgs<T>& a = *reinterpret_cast<DisArgs<T>*>(raw);
    if (threadIdx.x == 0) a = args;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double xl[D];
#pragma unroll
        for (int d = 0; d < D; ++d) xl[d] = x[i * D + d];
        out[i] = (double)term_value<T, TERM>(a, xl, rule);
    }
}

template <typename T>
__global__ void amplitude_kernel(const DisArgs<T> a, const double* __restrict__ r, const double* __restrict__ Y,
                                 int64_t n, double* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)amplitude(a, r[i], Y[i]);
}

// ===========================================================================
// Tensor Gauss-Legendre on the unit square, fine and half-order rules
// (custom_kernels/quadrature.py:14-58): one CTA per job, fixed-order reduction.

template <typename T, int TERM>
__global__ void gauss_legendre_kernel(const DisArgs<T>* __restrict__ args, InnerRule rule, GLRules gl,
                                      double* __restrict__ out)
{
    static_assert(term_dims(TERM) == 2, "tensor rule is used for the 2D terms");
    __shared__ __align__(16) unsigned char raw[sizeof(DisArgs<T>)];
    DisArgs<T>& a = *reinterpret_cast<DisArgs<T>*>(raw);
    if (threadIdx.x == 0) a = args[blockIdx.x];
    __shared__ double red[2][32];
    __syncthreads();
    double acc[2] = {0.0, 0.0};
#pragma unroll
    for (int which = 0; which < 2; ++which) {
        const int n = which == 0 ? gl.n_fine : gl.n_coarse;
        const double* xs = which == 0 ? gl.x_fine : gl.x_coarse;
        const double* ws = which == 0 ? gl.w_fine : gl.w_coarse;
        for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
            const int i0 = k / n, i1 = k % n;
            const double xl[2] = {xs[i0], xs[i1]};
            acc[which] += ws[i0] * ws[i1] * (double)term_value<T, TERM>(a, xl, rule);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int which = 0; which < 2; ++which) {
        double v = acc[which];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[which][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double f = 0.0, c = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            f += red[0][w];
            c += red[1][w];
        }
        out[2 * blockIdx.x + 0] = f;
        out[2 * blockIdx.x + 1] = ::fabs(f - c);
    }
}

// ===========================================================================
// Vegas

// partial layout per (job, block): [total, total2, hist[D][bins]] doubles and
// count[D][bins] int32 in a parallel array
// CTAs per SM the register bound aims at: the FP32 LO and dipole terms are latency-bound
// and run faster at four (64 registers); the qqbar-g terms keep three (80 registers),
// where the nested ones issue an instruction nearly every cycle and I1 gains nothing
// from a fourth CTA but spills.
template <typename T, int TERM>
constexpr int vegas_min_blocks()
{
    return sizeof(T) == 4 && TERM <= kTermDip2 ? 4 : 3;
}

template <typename T, int TERM>
__global__ void __launch_bounds__(kVegasThreads, (vegas_min_blocks<T, TERM>())) vegas_iteration_kernel(
    const DisArgs<T>* __restrict__ args, const SobolDirsArg* __restrict__ dirs, InnerRule rule,
    double* __restrict__ state, int state_stride, int bins, uint64_t offset, uint64_t samples, int blocks_per_job,
    double* __restrict__ partial, int32_t* __restrict__ counts)
{
    constexpr int D = term_dims(TERM);
    const int job = blockIdx.y;
    const double* st = state + (size_t)job * state_stride;
    if (st[D * (bins + 1) + kStConverged] != 0.0) return;  // uniform per job

    extern __shared__ __align__(16) unsigned char vsmem[];
    double* edges = reinterpret_cast<double*>(vsmem);                    // [D][bins+1]
    double* whist = edges + D * (bins + 1);                              // [warps][D*bins]
    int32_t* cnt = reinterpret_cast<int32_t*>(whist + (kVegasThreads / 32) * D * bins);  // [D*bins]
    __shared__ double red[2][kVegasThreads / 32];
    __shared__ uint32_t sst[D][30];
    __shared__ uint32_t ssh[D];

    const int warps = kVegasThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < D * (bins + 1); k += blockDim.x) edges[k] = st[k];
    for (int k = threadIdx.x; k < warps * D * bins; k += blockDim.x) whist[k] = 0.0;
    for (int k = threadIdx.x; k < D * bins; k += blockDim.x) cnt[k] = 0;
    const SobolDirsArg& sd = dirs[job];
    for (int k = threadIdx.x; k < D * 30; k += blockDim.x) sst[k / 30][k % 30] = sd.state[k / 30][k % 30];
    if (threadIdx.x < D) ssh[threadIdx.x] = sd.shift[threadIdx.x];
    __shared__ __align__(16) unsigned char raw[sizeof(DisArgs<T>)];
    DisArgs<T>& a = *reinterpret_cast<DisArgs<T>*>(raw);
    if (threadIdx.x == 0) a = args[job];
    __syncthreads();

    const uint64_t chunk = (samples + blocks_per_job - 1) / blocks_per_job;
    const uint64_t begin = (uint64_t)blockIdx.x * chunk;
    const uint64_t end = begin + chunk < samples ? begin + chunk : samples;
    double tot = 0.0, tot2 = 0.0;
    double* myhist = whist + warp * D * bins;
    const double fb = (double)bins;
    for (uint64_t base = begin; base < end; base += kVegasThreads) {
        const uint64_t i = base + threadIdx.x;
        const bool active = i < end;
        double xl[D];
        int bin[D];
        double inv_density = 1.0;
        if (active) {
            const uint64_t index = offset + i;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const double u = sobol_unit<double>(sobol_bits(sst[d], ssh[d], index), index);
                const double scaled = u * fb;
                int b = (int)floor(scaled);
                b = b > bins - 1 ? bins - 1 : b;
                const double frac = scaled - b;
                const double left = edges[d * (bins + 1) + b];
                const double width = edges[d * (bins + 1) + b + 1] - left;
                xl[d] = left + width * frac;
                inv_density *= fb * width;
                bin[d] = b;
            }
        }
        double w = 0.0;
        if (active) w = (double)term_value<T, TERM>(a, xl, rule) * inv_density;
        tot += w;
        tot2 += w * w;
        // deterministic warp histogram: lanes that share a bin add in lane order
        const unsigned mask = __ballot_sync(0xffffffffu, active);
        if (active) {
            const double aw = ::fabs(w);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const int key = d * bins + bin[d];
                const unsigned peers = __match_any_sync(mask, key);
                const int rank = __popc(peers & ((1u << lane) - 1u));
                const int last = __reduce_max_sync(mask, rank);
                for (int k = 0; k <= last; ++k) {
                    if (rank == k) myhist[key] += aw;
                    __syncwarp(mask);
                }
                atomicAdd(&cnt[key], 1);
            }
        }
    }
    // block reduction of the sums in warp order
    for (int o = 16; o > 0; o >>= 1) {
        tot += __shfl_down_sync(0xffffffffu, tot, o);
        tot2 += __shfl_down_sync(0xffffffffu, tot2, o);
    }
    if (lane == 0) {
        red[0][warp] = tot;
        red[1][warp] = tot2;
    }
    __syncthreads();
    const size_t pstride = 2 + (size_t)D * bins;
    double* out = partial + ((size_t)job * blocks_per_job + blockIdx.x) * pstride;
    int32_t* cout = counts + (size_t)job * D * bins;  // per-job bin counts, integer atomics
    if (threadIdx.x == 0) {
        double s = 0.0, s2 = 0.0;
        for (int w = 0; w < warps; ++w) {
            s += red[0][w];
            s2 += red[1][w];
        }
        out[0] = s;
        out[1] = s2;
    }
    for (int k = threadIdx.x; k < D * bins; k += blockDim.x) {
        double h = 0.0;
        for (int w = 0; w < warps; ++w) h += whist[w * D * bins + k];
        out[2 + k] = h;
        if (cnt[k]) atomicAdd(&cout[k], cnt[k]);
    }
}

// Sum the per-CTA partials of every job in a fixed order: grid (key chunks, jobs), one
// thread per key (the |w| histogram bins, then total and total^2), looping over the CTAs.
// Per job: sum the per-CTA partials [blocks][keys] over the CTAs.  Each thread takes one
// key and every kReduceSlices-th CTA row (four chains), and the slices of a key are added
// in slice order through shared memory, so the order is fixed; a warp reads 32 consecutive
// keys of a row.
constexpr int kReduceKeys = 32;
constexpr int kReduceSlices = 8;

__global__ void __launch_bounds__(kReduceKeys * kReduceSlices)
    vegas_reduce_kernel(const double* __restrict__ partial, int keys, int blocks_per_job, double* __restrict__ reduced)
{
    __shared__ double sums[kReduceSlices][kReduceKeys];
    const int job = blockIdx.y;
    const int kl = threadIdx.x % kReduceKeys, slice = threadIdx.x / kReduceKeys;
    const int k = blockIdx.x * kReduceKeys + kl;  // 0..keys-1 over [total, total2, hist...]
    double total = 0.0;
    if (k < keys) {
        const double* p = partial + (size_t)job * blocks_per_job * keys + k;
        constexpr int S = kReduceSlices;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int b = slice;
        for (; b + 3 * S < blocks_per_job; b += 4 * S) {
            a0 += p[(size_t)b * keys];
            a1 += p[(size_t)(b + S) * keys];
            a2 += p[(size_t)(b + 2 * S) * keys];
            a3 += p[(size_t)(b + 3 * S) * keys];
        }
        for (; b < blocks_per_job; b += S) a0 += p[(size_t)b * keys];
        total = (a0 + a1) + (a2 + a3);
    }
    sums[slice][kl] = total;
    __syncthreads();
    if (slice == 0 && k < keys) {
        double v = sums[0][kl];
        for (int q = 1; q < kReduceSlices; ++q) v += sums[q][kl];
        reduced[(size_t)job * keys + k] = v;
    }
}

// One CTA per job: adapt the grid (numerics/integration.py:804-866) from the reduced
// histogram and counts, update the combined estimate (:510-582), clear the counts.
__global__ void vegas_finalize_kernel(double* __restrict__ state, int state_stride, int D, int bins,
                                      uint64_t samples, const double* __restrict__ reduced,
                                      int32_t* __restrict__ counts, int warmup, int min_iterations,
                                      double epsrel, double epsabs)
{
    extern __shared__ double fsm[];
    double* smooth = fsm;               // [D*bins]
    double* cum = smooth + D * bins;    // [D*(bins+1)]
    double* ne = cum + D * (bins + 1);  // [D*(bins+1)]
    const int job = blockIdx.x;
    double* st = state + (size_t)job * state_stride;
    double* sc = st + D * (bins + 1);
    int32_t* c = counts + (size_t)job * D * bins;
    if (sc[kStConverged] != 0.0) return;
    const int keys = 2 + D * bins;
    const double* red = reduced + (size_t)job * keys;
    vegas::rebin(st, red + 2, c, D, bins, smooth, cum, ne);
    __syncthreads();
    for (int k = threadIdx.x; k < D * bins; k += blockDim.x) c[k] = 0;
    if (threadIdx.x == 0) {
        sc[kStEvals] += (double)samples;
        if (!warmup) vegas::combine(sc, red[0], red[1], (double)samples, min_iterations, epsrel, epsabs);
    }
}

__global__ void vegas_init_kernel(double* state, int state_stride, int D, int bins, int jobs, int keep_edges,
                                  int32_t* counts)
{
    const int job = blockIdx.x;
    if (job >= jobs) return;
    for (int k = threadIdx.x; k < D * bins; k += blockDim.x) counts[(size_t)job * D * bins + k] = 0;
    double* st = state + (size_t)job * state_stride;
    if (!keep_edges)
        for (int k = threadIdx.x; k < D * (bins + 1); k += blockDim.x) {
            const int b = k % (bins + 1);
            st[k] = b == bins ? 1.0 : (double)b / bins;
        }
    double* sc = st + D * (bins + 1);
    for (int k = threadIdx.x; k < kStSlots; k += blockDim.x) sc[k] = 0.0;
}

// ===========================================================================
// launchers

template <typename T, int TERM>
cudaError_t launch_points_t(const void* args, const InnerRule& rule, const double* x, int64_t n, double* out,
                            cudaStream_t stream)
{
    const int threads = 128;
    int64_t blocks = (n + threads - 1) / threads;
    blocks = blocks > 4096 ? 4096 : (blocks < 1 ? 1 : blocks);
    points_kernel<T, TERM><<<(unsigned)blocks, threads, 0, stream>>>(*static_cast<const DisArgs<T>*>(args), rule, x, n,
                                                                     out);
    return cudaGetLastError();
}

template <typename T, int TERM>
cudaError_t launch_gl_t(const void* args, int jobs, const InnerRule& rule, const GLRules& gl, double* out,
                        cudaStream_t stream)
{
    if constexpr (term_dims(TERM) == 2) {
        gauss_legendre_kernel<T, TERM><<<jobs, 256, 0, stream>>>(static_cast<const DisArgs<T>*>(args), rule, gl, out);
        return cudaGetLastError();
    } else {
        return cudaErrorInvalidValue;
    }
}

template <typename T, int TERM>
cudaError_t launch_vegas_round_t(const VegasLaunch& L, cudaStream_t stream)
{
    constexpr int D = term_dims(TERM);
    const size_t smem = sizeof(double) * (D * (L.bins + 1) + (kVegasThreads / 32) * D * L.bins) +
                        sizeof(int32_t) * D * L.bins;
    auto kern = vegas_iteration_kernel<T, TERM>;
    cudaError_t e = raise_dynamic_smem((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(L.blocks_per_job, L.jobs);
    kern<<<grid, kVegasThreads, smem, stream>>>(static_cast<const DisArgs<T>*>(L.args), L.dirs, *L.rule, L.state,
                                                L.state_stride, L.bins, L.offset, L.samples, L.blocks_per_job,
                                                L.partial, L.counts);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int keys = 2 + D * L.bins;
    dim3 rgrid((keys + kReduceKeys - 1) / kReduceKeys, L.jobs);
    vegas_reduce_kernel<<<rgrid, kReduceKeys * kReduceSlices, 0, stream>>>(L.partial, keys, L.blocks_per_job,
                                                                           L.reduced);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t fsmem = sizeof(double) * (D * L.bins + 2 * D * (L.bins + 1));
    e = raise_dynamic_smem((const void*)vegas_finalize_kernel, fsmem);
    if (e != cudaSuccess) return e;
    vegas_finalize_kernel<<<L.jobs, 128, fsmem, stream>>>(L.state, L.state_stride, D, L.bins, L.samples, L.reduced,
                                                          L.counts, L.warmup, L.min_iterations, L.epsrel, L.epsabs);
    return cudaGetLastError();
}

#define NLO_DIS_DISPATCH(FN, ...)                                                  \
    switch (term) {                                                                \
        case kTermLO: return FN<T, kTermLO>(__VA_ARGS__);                          \
        case kTermDip0: return FN<T, kTermDip0>(__VA_ARGS__);                      \
        case kTermDip1: return FN<T, kTermDip1>(__VA_ARGS__);                      \
        case kTermDip2: return FN<T, kTermDip2>(__VA_ARGS__);                      \
        case kTermI1: return FN<T, kTermI1>(__VA_ARGS__);                          \
        case kTermI2: return FN<T, kTermI2>(__VA_ARGS__);                          \
        case kTermI3: return FN<T, kTermI3>(__VA_ARGS__);                          \
        case kTermI2N: return FN<T, kTermI2N>(__VA_ARGS__);                        \
        case kTermI3N: return FN<T, kTermI3N>(__VA_ARGS__);                        \
        default: return cudaErrorInvalidValue;                                     \
    }

template <typename T>
cudaError_t launch_points_typed(int term, const void* args, const InnerRule& rule, const double* x, int64_t n,
                                double* out, cudaStream_t stream)
{
    NLO_DIS_DISPATCH(launch_points_t, args, rule, x, n, out, stream)
}

template <typename T>
cudaError_t launch_gl_typed(int term, const void* args, int jobs, const InnerRule& rule, const GLRules& gl,
                            double* out, cudaStream_t stream)
{
    switch (term) {
        case kTermLO: return launch_gl_t<T, kTermLO>(args, jobs, rule, gl, out, stream);
        case kTermDip0: return launch_gl_t<T, kTermDip0>(args, jobs, rule, gl, out, stream);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t launch_vegas_round_typed(int term, const VegasLaunch& L, cudaStream_t stream)
{
    NLO_DIS_DISPATCH(launch_vegas_round_t, L, stream)
}

}  // namespace dis

cudaError_t dis_launch_table_prepare(const double* r, const double* y, const double* N, int nr, int ny, double y0,
                                     int interp, double* table, cudaStream_t stream)
{
    int blocks = (nr * ny + 255) / 256;
    blocks = blocks > 1024 ? 1024 : (blocks < 1 ? 1 : blocks);
    dis::table_prepare_kernel<<<blocks, 256, 0, stream>>>(r, y, N, nr, ny, y0, interp, table);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int64_t items = (int64_t)ny * (nr - 1);
    int64_t local_blocks = (items + 255) / 256;
    local_blocks = local_blocks > 2048 ? 2048 : (local_blocks < 1 ? 1 : local_blocks);
    dis::table_local_kernel<<<(unsigned)local_blocks, 256, 0, stream>>>(table, nr, ny);
    return cudaGetLastError();
}

cudaError_t dis_launch_table_initialize(double* table, int nr, int ny, double Y, cudaStream_t stream)
{
    const size_t smem = sizeof(double) * 3 * (size_t)nr;
    cudaError_t e = raise_dynamic_smem((const void*)dis::table_initialize_kernel, smem);
    if (e != cudaSuccess) return e;
    dis::table_initialize_kernel<<<1, 256, smem, stream>>>(table, nr, ny, Y);
    return cudaGetLastError();
}

cudaError_t dis_launch_points(int precision, int term, const void* args, const dis::InnerRule& rule, const double* x,
                              int64_t n, double* out, cudaStream_t stream)
{
    return precision == NLO_PRECISION_FP64 ? dis::launch_points_typed<double>(term, args, rule, x, n, out, stream)
                                           : dis::launch_points_typed<float>(term, args, rule, x, n, out, stream);
}

cudaError_t dis_launch_amplitude(int precision, const void* args, const double* r, const double* Y, int64_t n,
                                 double* out, cudaStream_t stream)
{
    int64_t blocks = (n + 255) / 256;
    blocks = blocks > 4096 ? 4096 : (blocks < 1 ? 1 : blocks);
    if (precision == NLO_PRECISION_FP64)
        dis::amplitude_kernel<double><<<(unsigned)blocks, 256, 0, stream>>>(
            *static_cast<const dis::DisArgs<double>*>(args), r, Y, n, out);
    else
        dis::amplitude_kernel<float><<<(unsigned)blocks, 256, 0, stream>>>(
            *static_cast<const dis::DisArgs<float>*>(args), r, Y, n, out);
    return cudaGetLastError();
}

cudaError_t dis_launch_gl(int precision, int term, const void* args, int jobs, const dis::InnerRule& rule,
                          const dis::GLRules& gl, double* out, cudaStream_t stream)
{
    return precision == NLO_PRECISION_FP64 ? dis::launch_gl_typed<double>(term, args, jobs, rule, gl, out, stream)
                                           : dis::launch_gl_typed<float>(term, args, jobs, rule, gl, out, stream);
}

cudaError_t dis_launch_vegas_init(double* state, int state_stride, int D, int bins, int jobs, int keep_edges,
                                  int32_t* counts, cudaStream_t stream)
{
    dis::vegas_init_kernel<<<jobs, 128, 0, stream>>>(state, state_stride, D, bins, jobs, keep_edges, counts);
    return cudaGetLastError();
}

cudaError_t dis_launch_reduce_finalize(int D, int bins, int jobs, int blocks_per_job, const double* partial,
                                       double* reduced, int32_t* counts, double* state, int state_stride,
                                       uint64_t samples, int warmup, int min_iterations, double epsrel, double epsabs,
                                       cudaStream_t stream)
{
    const int keys = 2 + D * bins;
    dim3 rgrid((keys + dis::kReduceKeys - 1) / dis::kReduceKeys, jobs);
    dis::vegas_reduce_kernel<<<rgrid, dis::kReduceKeys * dis::kReduceSlices, 0, stream>>>(partial, keys,
                                                                                       blocks_per_job, reduced);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t fsmem = sizeof(double) * (D * bins + 2 * D * (bins + 1));
    e = raise_dynamic_smem((const void*)dis::vegas_finalize_kernel, fsmem);
    if (e != cudaSuccess) return e;
    dis::vegas_finalize_kernel<<<jobs, 128, fsmem, stream>>>(state, state_stride, D, bins, samples, reduced, counts,
                                                               warmup, min_iterations, epsrel, epsabs);
    return cudaGetLastError();
}

cudaError_t vegas_launch_reduce(const double* partial, int keys, int blocks_per_job, int jobs, double* reduced,
                                cudaStream_t stream)
{
    dim3 rgrid((keys + dis::kReduceKeys - 1) / dis::kReduceKeys, jobs);
    dis::vegas_reduce_kernel<<<rgrid, dis::kReduceKeys * dis::kReduceSlices, 0, stream>>>(partial, keys,
                                                                                       blocks_per_job, reduced);
    return cudaGetLastError();
}

cudaError_t dis_launch_vegas_round(int precision, int term, const dis::VegasLaunch& L, cudaStream_t stream)
{
    return precision == NLO_PRECISION_FP64 ? dis::launch_vegas_round_typed<double>(term, L, stream)
                                           : dis::launch_vegas_round_typed<float>(term, L, stream);
}

}  // namespace nlo
