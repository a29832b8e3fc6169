// Right-hand-side assembly and the rapidity step (FP64).
//
// dN/dY = K1 + (K2+Kf) with non-finite values replaced by 0 (bk/evolution.py:329-351);
// inactive parents carry zeros because their K1 and K2+Kf entries are zeroed.
// A stage input is N + sum_k c_k k_k; the final combination of a step optionally
// clamps to [0,1] (FORCE_POSITIVE_N, bk/evolution.py:150-151) and flags
// non-finite values in a status word (bk/evolution.py:152-153 raises on the host).

#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"

namespace nlo {

namespace {

__global__ void assemble_kernel(const double* __restrict__ k1, const double* __restrict__ k2kf, int n,
                                double inv_samples, double* __restrict__ dndy, double* __restrict__ k2kf_total)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double nlo = (k2kf[3 * i] + k2kf[3 * i + 1]) * inv_samples;
    double v = k1[i] + nlo;
    if (!isfinite(v)) v = 0.0;
    dndy[i] = v;
    if (k2kf_total) k2kf_total[i] = nlo;
}

struct StageArgs {
    const double* k[4];
    double c[4];
    int nk;
};

__global__ void axpy_stage_kernel(const double* __restrict__ N, StageArgs a, int n, double* __restrict__ out,
                                  int clamp, uint32_t* __restrict__ status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = N[i];
    for (int j = 0; j < a.nk; ++j) v += a.c[j] * a.k[j][i];
    if (clamp) v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
    if (status && !isfinite(v)) atomicOr(status, (uint32_t)kStatusNonFinite);
    out[i] = v;
}

}  // namespace

cudaError_t launch_assemble(const double* k1, const double* k2kf, int points, double inv_samples, double* dndy,
                            double* k2kf_total, cudaStream_t stream)
{
    assemble_kernel<<<(points + 255) / 256, 256, 0, stream>>>(k1, k2kf, points, inv_samples, dndy, k2kf_total);
    return cudaGetLastError();
}

cudaError_t launch_axpy_stage(const double* N, const double* const* k, const double* coef, int nk, int points,
                              double* out, int clamp, uint32_t* status, cudaStream_t stream)
{
    StageArgs a;
    a.nk = nk;
    for (int j = 0; j < 4; ++j) {
        a.k[j] = j < nk ? k[j] : nullptr;
        a.c[j] = j < nk ? coef[j] : 0.0;
    }
    axpy_stage_kernel<<<(points + 255) / 256, 256, 0, stream>>>(N, a, points, out, clamp, status);
    return cudaGetLastError();
}

}  // namespace nlo
