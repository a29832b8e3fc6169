// Log-log natural cubic splines of the evolving amplitude (FP64), the active
// parent list, and the device Sobol draw.
//
// Spline: restates numerics/interpolation.py:10-121 (natural cubic spline with a
// Thomas solve, log-log table with -40 for non-positive values) for the two
// evolution rows of bk/evolution.py:548-560: log N with N clamped to [0,1], and
// log S with S = 1 - N clamped to [0,1], evaluated as log1p(-N) so that S close to
// 1 keeps the relative precision of N.  One CTA per row pair; the two Thomas
// sweeps run concurrently in two warps.

#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "sobol.cuh"

namespace nlo {

// factor: [2][n] = 1/denominator and upper coefficient of the Thomas sweep for
// the natural-spline system on the knots log r (it depends on the grid only).
// With compute_factor set, thread 0 forms it first (and stores it for later calls).
// One CTA per set (blockIdx.x): row N.at(set), tables at out + set * spline_doubles(n), its own
// factorisation copy at factor + set * 2n.
__global__ void __launch_bounds__(256) splines_kernel(const double* __restrict__ r, RowsArg rows,
                                                      int n, int force_positive, double* __restrict__ factor,
                                                      int compute_factor, double* __restrict__ out)
{
    const double* __restrict__ N = rows.at(blockIdx.x);
    factor += (size_t)blockIdx.x * 2 * n;
    out += (size_t)blockIdx.x * spline_doubles(n);
    extern __shared__ double smem[];
    double* x = smem;             // [n]
    double* y = x + n;            // [2][n]
    double* rhs = y + 2 * n;      // [2][n]
    double* sol = rhs + 2 * n;    // [2][n]
    double* inv_den = sol + 2 * n;  // [n]
    double* up = inv_den + n;       // [n]
    const int m = n - 2;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        x[i] = log(r[i]);
        out[i] = x[i];
        const double v = N[i];
        // log N row: N > 1 -> 1; force_positive: N < 0 -> 0
        double vn = v > 1.0 ? 1.0 : v;
        if (force_positive && vn < 0.0) vn = 0.0;
        y[i] = vn > 0.0 ? log(vn) : kMinLog;
        // log S row: S = 1 - N; S < 0 -> 0; force_positive: S > 1 -> 1
        double ns = v;
        if (force_positive && ns < 0.0) ns = 0.0;
        y[n + i] = ns < 1.0 ? log1p(-ns) : kMinLog;
    }
    __syncthreads();
    for (int item = threadIdx.x; item < 2 * m; item += blockDim.x) {
        const int row = item / m, i = item - row * m;
        const double* yy = y + row * n;
        rhs[row * n + i] =
            6.0 * ((yy[i + 2] - yy[i + 1]) / (x[i + 2] - x[i + 1]) - (yy[i + 1] - yy[i]) / (x[i + 1] - x[i]));
    }
    if (compute_factor && threadIdx.x == 0 && m >= 1) {
        // denominators of the forward sweep (interpolation.py:124-149)
        double d = 2.0 * ((x[1] - x[0]) + (x[2] - x[1]));
        factor[0] = 1.0 / d;
        for (int i = 1; i < m; ++i) {
            const double upper_prev = (x[i + 1] - x[i]) * factor[i - 1];
            factor[n + i - 1] = upper_prev;
            d = 2.0 * ((x[i + 1] - x[i]) + (x[i + 2] - x[i + 1])) - (x[i + 1] - x[i]) * upper_prev;
            factor[i] = 1.0 / d;
        }
    }
    __syncthreads();
    // The forward sweep s_i = (b_i - h_i s_{i-1}) / d_i as s_i = c_i + a_i s_{i-1} with
    // c_i = b_i / d_i and a_i = -h_i / d_i formed in parallel, so the sequential chain is
    // one FMA a step whose operands load ahead of it; the back substitution likewise
    // with the negated upper diagonal.
    for (int item = threadIdx.x; item < 2 * m; item += blockDim.x) {
        const int row = item / m, i = item - row * m;
        rhs[row * n + i] *= factor[i];
        if (row == 0) {
            inv_den[i] = i > 0 ? -(x[i + 1] - x[i]) * factor[i] : 0.0;
            up[i] = i < m - 1 ? -factor[n + i] : 0.0;
        }
    }
    __syncthreads();
    // warp 0 solves row 0, warp 1 row 1
    if ((threadIdx.x & 31) == 0 && threadIdx.x < 64 && m >= 1) {
        const int row = threadIdx.x >> 5;
        const double* c = rhs + row * n;
        double* s = sol + row * n;
        double prev = c[0];
        s[0] = prev;
#pragma unroll 8
        for (int i = 1; i < m; ++i) {
            prev = fma(inv_den[i], prev, c[i]);
            s[i] = prev;
        }
        double next = prev;
#pragma unroll 8
        for (int i = m - 2; i >= 0; --i) {
            next = fma(up[i], next, s[i]);
            s[i] = next;
        }
    }
    __syncthreads();
    for (int item = threadIdx.x; item < 2 * (n - 1); item += blockDim.x) {
        const int row = item / (n - 1);
        const int i = item - row * (n - 1);
        const double* yy = y + row * n;
        const double* s = sol + row * n;
        const double h = x[i + 1] - x[i];
        const double sl = i == 0 ? 0.0 : s[i - 1];
        const double sr = i == n - 2 ? 0.0 : s[i];
        double* c = out + n + (size_t)row * 4 * (n - 1) + 4 * (size_t)i;
        c[0] = yy[i];
        c[1] = (yy[i + 1] - yy[i]) / h - h * (2.0 * sl + sr) / 6.0;
        c[2] = sl / 2.0;
        c[3] = (sr - sl) / (6.0 * h);
    }
}

// Active parents: index > 0 and N <= 0.99999 (bk/evolution.py:501), compacted in
// index order by a ballot scan, one CTA per set (blockIdx.x).
__global__ void __launch_bounds__(1024) active_kernel(RowsArg rows, int n, int shard, int shards,
                                                      int32_t* __restrict__ active, int32_t* __restrict__ count)
{
    const double* __restrict__ N = rows.at(blockIdx.x);
    active += (size_t)blockIdx.x * n;
    count += blockIdx.x;
    __shared__ int warp_counts[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int start = 0; start < n; start += blockDim.x) {
        const int i = start + threadIdx.x;
        const bool on = i < n && i > 0 && N[i] <= 0.99999 && i % shards == shard;
        const unsigned mask = __ballot_sync(0xffffffffu, on);
        if (lane == 0) warp_counts[warp] = __popc(mask);
        __syncthreads();
        int offset = base;
        for (int w = 0; w < warp; ++w) offset += warp_counts[w];
        if (on) active[offset + __popc(mask & ((1u << lane) - 1u))] = i;
        __syncthreads();
        if (threadIdx.x == 0) {
            int total = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) total += warp_counts[w];
            base += total;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = base;
}

template <typename T>
__global__ void sobol_draw_kernel(SobolDirsArg dirs, uint64_t offset, uint64_t n, T* __restrict__ out)
{
    const int d = dirs.dims;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t index = offset + k;
        for (int j = 0; j < d; ++j) {
            const uint32_t bits = sobol_bits(dirs.state[j], dirs.shift[j], index);
            out[k * d + j] = sobol_unit<T>(bits, index);
        }
    }
}

cudaError_t launch_splines(const double* r, const RowsArg& N, int n, int sets, int force_positive, double* factor,
                           int compute_factor, double* out, cudaStream_t stream)
{
    const size_t smem = sizeof(double) * 9 * (size_t)n;
    if (smem > 48 * 1024) {
        cudaError_t e = raise_dynamic_smem((const void*)splines_kernel, smem);
        if (e != cudaSuccess) return e;
    }
    splines_kernel<<<sets, 256, smem, stream>>>(r, N, n, force_positive, factor, compute_factor, out);
    return cudaGetLastError();
}

cudaError_t launch_active(const RowsArg& N, int n, int sets, int shard, int shards, int32_t* active, int32_t* count,
                          cudaStream_t stream)
{
    active_kernel<<<sets, 1024, 0, stream>>>(N, n, shard, shards, active, count);
    return cudaGetLastError();
}

cudaError_t launch_sobol(const SobolDirsArg& dirs, uint64_t offset, uint64_t n, int precision, void* out,
                         cudaStream_t stream)
{
    const int threads = 256;
    uint64_t blocks64 = (n + threads - 1) / threads;
    const int blocks = (int)(blocks64 > 65535 ? 65535 : (blocks64 == 0 ? 1 : blocks64));
    if (precision == NLO_PRECISION_FP64)
        sobol_draw_kernel<double><<<blocks, threads, 0, stream>>>(dirs, offset, n, (double*)out);
    else
        sobol_draw_kernel<float><<<blocks, threads, 0, stream>>>(dirs, offset, n, (float*)out);
    return cudaGetLastError();
}

}  // namespace nlo
