// Tabulated initial condition on the device: the natural cubic spline of ICDataFile
// (bk/initial_conditions.py:38-91) through the file's (r, N) rows, fitted and evaluated
// here so that a 30,000-row table never passes through the host.
//
// The fit follows NaturalCubicSpline (numerics/interpolation.py:13-48) and its Thomas
// solve (:124-149) operation for operation in FP64, so the coefficients are the
// reference's bit for bit: h_i = x_{i+1} - x_i, the interior system with diagonal
// 2 (h_i + h_{i+1}), off-diagonal h_{i+1} and right-hand side 6 ((y_{i+2} - y_{i+1})/h_{i+1}
// - (y_{i+1} - y_i)/h_i), forward elimination and back substitution, then
// b = dy/h - h (2 M_i + M_{i+1})/6, c = M_i/2, d = (M_{i+1} - M_i)/(6 h).  The two sweeps
// are a chain of dependent divisions and run in one thread (milliseconds for 30,000 rows,
// once per evolution); everything else is parallel.
//
// Buffer (nlo_ic_spline_doubles(n)): x[n] | a[n-1] | b[n-1] | c[n-1] | d[n-1].  During
// the fit b holds h, c the elimination multipliers and d the right-hand side / solution.

#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"

namespace nlo {
namespace {

constexpr int kIcThreads = 1024;

__global__ void __launch_bounds__(kIcThreads) ic_fit_kernel(const double* __restrict__ r, const double* __restrict__ N,
                                                            int n, double* __restrict__ spline)
{
    double* x = spline;
    double* a = x + n;
    double* b = a + (n - 1);
    double* c = b + (n - 1);
    double* d = c + (n - 1);
    const int m = n - 2;  // interior second derivatives
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = r[i];
    for (int i = threadIdx.x; i < n - 1; i += blockDim.x) {
        a[i] = N[i];
        b[i] = r[i + 1] - r[i];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x)
        d[i] = 6.0 * ((N[i + 2] - N[i + 1]) / b[i + 1] - (N[i + 1] - N[i]) / b[i]);
    __syncthreads();
    if (threadIdx.x == 0) {
        // diagonal_i = 2 (h_i + h_{i+1}), off_i = h_{i+1}.  The chain runs through the
        // divisions; the next iteration's h and right-hand side are loaded one step ahead
        // so that their latency hides behind it.
        if (m == 1) {
            d[0] = d[0] / (2.0 * (b[0] + b[1]));
        } else {
            double upper = b[1] / (2.0 * (b[0] + b[1]));
            double sol = d[0] / (2.0 * (b[0] + b[1]));
            c[0] = upper;
            d[0] = sol;
            double h_i = b[1], h_next = b[2], rhs = d[1];
            for (int i = 1; i < m; ++i) {
                const double h_after = i + 2 < n - 1 ? b[i + 2] : 0.0;
                const double rhs_after = i + 1 < m ? d[i + 1] : 0.0;
                const double den = 2.0 * (h_i + h_next) - h_i * upper;
                if (i < m - 1) {
                    upper = h_next / den;
                    c[i] = upper;
                }
                sol = (rhs - h_i * sol) / den;
                d[i] = sol;
                h_i = h_next;
                h_next = h_after;
                rhs = rhs_after;
            }
            double next = d[m - 1];
            double cu = m - 2 >= 0 ? c[m - 2] : 0.0, dv = m - 2 >= 0 ? d[m - 2] : 0.0;
            for (int i = m - 2; i >= 0; --i) {
                const double cu_after = i > 0 ? c[i - 1] : 0.0;
                const double dv_after = i > 0 ? d[i - 1] : 0.0;
                next = dv - cu * next;
                d[i] = next;
                cu = cu_after;
                dv = dv_after;
            }
        }
    }
    __syncthreads();
    // second derivatives M_0 = 0, M_{i+1} = d[i], M_{n-1} = 0: c_i = M_i / 2 first ...
    for (int i = threadIdx.x; i < n - 1; i += blockDim.x) c[i] = i == 0 ? 0.0 : d[i - 1] / 2.0;
    __syncthreads();
    // ... then b and d from M_i = 2 c_i (exact) and M_{i+1}
    for (int i = threadIdx.x; i < n - 1; i += blockDim.x) {
        const double h = b[i];
        const double Mi = 2.0 * c[i];
        const double Mj = i + 1 < n - 1 ? 2.0 * c[i + 1] : 0.0;
        b[i] = (N[i + 1] - N[i]) / h - h * (2.0 * Mi + Mj) / 6.0;
        d[i] = (Mj - Mi) / (6.0 * h);
    }
}

// ICDataFile.dipole_amplitude (bk/initial_conditions.py:86-90): 0 below the first r, 1
// above the last, the spline in between (interval searchsorted(x, r, right) - 1 clamped).
__global__ void ic_evaluate_kernel(const double* __restrict__ spline, int n, const double* __restrict__ r, int64_t m,
                                   double* __restrict__ out)
{
    const double* x = spline;
    const double* a = x + n;
    const double* b = a + (n - 1);
    const double* c = b + (n - 1);
    const double* d = c + (n - 1);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const double v = r[k];
        if (v < x[0]) {
            out[k] = 0.0;
            continue;
        }
        if (v > x[n - 1]) {
            out[k] = 1.0;
            continue;
        }
        int lo = 0, hi = n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (x[mid] <= v) lo = mid + 1; else hi = mid;
        }
        int i = lo - 1;
        i = i < 0 ? 0 : (i > n - 2 ? n - 2 : i);
        const double dx = v - x[i];
        out[k] = a[i] + dx * (b[i] + dx * (c[i] + dx * d[i]));
    }
}

}  // namespace
}  // namespace nlo

extern "C" {

size_t nlo_ic_spline_doubles(int32_t n) { return n < 3 ? 0 : (size_t)5 * n - 4; }

int nlo_ic_spline(const double* r, const double* N, int32_t n, double* spline, void* stream)
{
    if (!r || !N || !spline) return nlo::set_last_error(NLO_ERR_INVALID, "nlo_ic_spline: NULL buffer");
    if (n < 3) return nlo::set_last_error(NLO_ERR_INVALID, "a cubic spline requires at least three points");
    nlo::ic_fit_kernel<<<1, nlo::kIcThreads, 0, static_cast<cudaStream_t>(stream)>>>(r, N, n, spline);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NLO_OK : nlo::set_last_error(NLO_ERR_CUDA, cudaGetErrorString(e));
}

int nlo_ic_evaluate(const double* spline, int32_t n, const double* r, int64_t m, double* out, void* stream)
{
    if (!spline || (m > 0 && (!r || !out))) return nlo::set_last_error(NLO_ERR_INVALID, "nlo_ic_evaluate: NULL buffer");
    if (n < 3 || m < 0) return nlo::set_last_error(NLO_ERR_INVALID, "nlo_ic_evaluate: bad sizes");
    if (m == 0) return NLO_OK;
    int64_t blocks = (m + 255) / 256;
    blocks = blocks > 4096 ? 4096 : blocks;
    nlo::ic_evaluate_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(spline, n, r, m, out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NLO_OK : nlo::set_last_error(NLO_ERR_CUDA, cudaGetErrorString(e));
}

}  // extern "C"
