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

// Several parameter sets: blockIdx.y is the set.
__global__ void assemble_sets_kernel(const double* __restrict__ k1, const double* __restrict__ k2kf, int n,
                                     const SetTable* __restrict__ table, double* __restrict__ dndy)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (i >= n) return;
    const double* q = k2kf + 3 * ((size_t)s * n + i);
    const double nlo = (q[0] + q[1]) * table->inv[s];
    double v = k1[(size_t)s * n + i] + nlo;
    if (!isfinite(v)) v = 0.0;
    dndy[(size_t)s * n + i] = v;
}

__global__ void axpy_sets_kernel(RowsArg N, StageArgs a, int n, RowsArg out, int clamp, uint32_t* __restrict__ status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (i >= n) return;
    double v = N.at(s)[i];
    for (int j = 0; j < a.nk; ++j) v += a.c[j] * a.k[j][(size_t)s * n + i];
    if (clamp) v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
    if (status && !isfinite(v)) atomicOr(status + s, (uint32_t)kStatusNonFinite);
    out.at(s)[i] = v;
}

struct SetupArg {
    double* rows[kMaxSets];
    uint32_t samples[kMaxSets];
    int16_t slot_set[kMaxSlots];
    int sets, slots, nlo;
};
static_assert(sizeof(SetupArg) <= 4096, "the set table travels as a kernel parameter");

// Sobol directions of up to kDirsPerLaunch sets per launch (a large kernel parameter).
constexpr int kDirsPerLaunch = 48;
struct DirsArg {
    int first, count;
    uint32_t words[kDirsPerLaunch][kSetDirsWords];
};
static_assert(sizeof(DirsArg) <= 32000, "within the kernel parameter limit of sm_70 and later");

__global__ void sets_dirs_kernel(DirsArg a, SetTable* __restrict__ t)
{
    for (int i = threadIdx.x; i < a.count * kSetDirsWords; i += blockDim.x)
        t->dirs[a.first + i / kSetDirsWords][i % kSetDirsWords] = a.words[i / kSetDirsWords][i % kSetDirsWords];
}

__global__ void sets_setup_kernel(SetupArg a, SetTable* __restrict__ t)
{
    const int i = threadIdx.x;
    if (i < kMaxSets) {
        t->rows[i] = i < a.sets ? a.rows[i] : nullptr;
        t->samples[i] = i < a.sets ? a.samples[i] : 0u;
        t->inv[i] = i < a.sets && a.nlo && a.samples[i] > 0 ? 1.0 / (double)a.samples[i] : 0.0;
    }
    if (i < kMaxSlots) t->slot_set[i] = i < a.slots ? (int32_t)a.slot_set[i] : -1;
    __syncthreads();
    if (i < a.slots && t->slot_set[i] >= 0) t->set_slot[t->slot_set[i]] = i;
}

}  // namespace

cudaError_t launch_sets_setup(double* const* rows, const int64_t* samples, const int32_t* slot_set,
                              const SobolDirsArg* const* dirs, int sets, int slots, bool nlo, SetTable* table,
                              cudaStream_t stream)
{
    if (sets < 1 || sets > kMaxSets || slots < sets || slots > kMaxSlots) return cudaErrorInvalidValue;
    SetupArg a;
    for (int i = 0; i < kMaxSets; ++i) {
        a.rows[i] = i < sets ? rows[i] : nullptr;
        a.samples[i] = i < sets ? (uint32_t)samples[i] : 0u;
    }
    for (int i = 0; i < kMaxSlots; ++i) a.slot_set[i] = (int16_t)(i < slots ? slot_set[i] : -1);
    a.sets = sets;
    a.slots = slots;
    a.nlo = nlo ? 1 : 0;
    sets_setup_kernel<<<1, (kMaxSlots + 31) / 32 * 32, 0, stream>>>(a, table);
    cudaError_t e = cudaGetLastError();
    for (int first = 0; first < sets && e == cudaSuccess; first += kDirsPerLaunch) {
        DirsArg d;
        d.first = first;
        d.count = sets - first < kDirsPerLaunch ? sets - first : kDirsPerLaunch;
        for (int k = 0; k < d.count; ++k) {
            const SobolDirsArg& src = *dirs[first + k];
            for (int j = 0; j < 4; ++j) {
                for (int b = 0; b < 30; ++b) d.words[k][30 * j + b] = src.state[j][b];
                d.words[k][120 + j] = src.shift[j];
            }
        }
        sets_dirs_kernel<<<1, 256, 0, stream>>>(d, table);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_assemble_sets(const double* k1, const double* k2kf, int points, int sets, const SetTable* table,
                                 double* dndy, cudaStream_t stream)
{
    assemble_sets_kernel<<<dim3((points + 255) / 256, sets), 256, 0, stream>>>(k1, k2kf, points, table, dndy);
    return cudaGetLastError();
}

cudaError_t launch_axpy_sets(const RowsArg& N, const double* const* k, const double* coef, int nk, int points,
                             int sets, const RowsArg& out, int clamp, uint32_t* status, cudaStream_t stream)
{
    StageArgs a;
    a.nk = nk;
    for (int j = 0; j < 4; ++j) {
        a.k[j] = j < nk ? k[j] : nullptr;
        a.c[j] = j < nk ? coef[j] : 0.0;
    }
    axpy_sets_kernel<<<dim3((points + 255) / 256, sets), 256, 0, stream>>>(N, a, points, out, clamp, status);
    return cudaGetLastError();
}

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
