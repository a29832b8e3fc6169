// Vegas for an integrand the caller evaluates: the vegas() entry point of
// numerics/integration.py:120-589 for any function of a batch of points.  The library owns
// the sampling and the bookkeeping on the device; the caller owns the integrand:
//
//   nlo_vegas_begin       uniform grid (or the caller's kept grid), cleared sums;
//   nlo_vegas_sample      scrambled Sobol points (indices offset..) mapped through the grid:
//                         box points x[n][dims], the weight factor volume x prod(bins width),
//                         the bin of every coordinate;
//   (caller)              f(x) for the batch;
//   nlo_vegas_accumulate  w = f x factor into the round's sums of w, w^2 and the |w|
//                         histograms (per-CTA partials, added in a fixed order);
//   nlo_vegas_end_round   the grid re-binning and, after a warm-up round, the estimate's
//                         inverse-variance combination and convergence test
//                         (vegas_common.cuh, the code of the BK and DIS integrals).
//
// A coordinate u of a Sobol point gives the bin floor(u bins) and the fraction u bins - bin.
#include <cuda_runtime.h>

#include <string>

#include "internal.h"
#include "sobol.cuh"
#include "vegas_common.cuh"

namespace nlo {

namespace {

using namespace vegas;

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxDims = 8;
constexpr int kBlocks = 148;  // partial rows per batch

// Workspace: round sums [2 + D*bins] | batch partials [kBlocks][2 + D*bins] |
// batch sums [2 + D*bins] | counts [D*bins] int32.
struct GenericBuffers {
    double* round;
    double* partial;
    double* batch;
    int32_t* counts;
};

size_t keys_of(int dims, int bins) { return 2 + (size_t)dims * bins; }

GenericBuffers carve_generic(void* ws, int dims, int bins)
{
    const size_t keys = keys_of(dims, bins);
    GenericBuffers b;
    b.round = static_cast<double*>(ws);
    b.partial = b.round + keys;
    b.batch = b.partial + keys * kBlocks;
    b.counts = reinterpret_cast<int32_t*>(b.batch + keys);
    return b;
}

__global__ void begin_kernel(double* state, int dims, int bins, int keep_edges, double* round, int32_t* counts)
{
    for (int k = threadIdx.x; k < dims * bins; k += blockDim.x) counts[k] = 0;
    for (int k = threadIdx.x; k < 2 + dims * bins; k += blockDim.x) round[k] = 0.0;
    if (!keep_edges)
        for (int k = threadIdx.x; k < dims * (bins + 1); k += blockDim.x) {
            const int b = k % (bins + 1);
            state[k] = b == bins ? 1.0 : (double)b / bins;
        }
    double* sc = state + dims * (bins + 1);
    for (int k = threadIdx.x; k < kStSlots; k += blockDim.x) sc[k] = 0.0;
}

struct BoxArg {
    double lower[kMaxDims], width[kMaxDims];
    double volume;
};

__global__ void sample_kernel(SobolDirsArg dirs, uint64_t offset, uint64_t n, int dims, int bins,
                              const double* __restrict__ state, BoxArg box, double* __restrict__ x,
                              double* __restrict__ factor, int32_t* __restrict__ bin)
{
    extern __shared__ double edges[];  // [dims][bins+1]
    for (int k = threadIdx.x; k < dims * (bins + 1); k += blockDim.x) edges[k] = state[k];
    __syncthreads();
    const double fb = (double)bins;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t index = offset + i;
        double inv_density = 1.0;
        for (int d = 0; d < dims; ++d) {
            const double u = sobol_unit<double>(sobol_bits(dirs.state[d], dirs.shift[d], index), index);
            const double scaled = u * fb;
            int b = (int)floor(scaled);
            b = b > bins - 1 ? bins - 1 : b;
            const double frac = scaled - b;
            const double left = edges[d * (bins + 1) + b];
            const double w = edges[d * (bins + 1) + b + 1] - left;
            x[i * dims + d] = box.lower[d] + box.width[d] * (left + w * frac);
            inv_density *= fb * w;
            bin[i * dims + d] = b;
        }
        factor[i] = box.volume * inv_density;
    }
}

__global__ void __launch_bounds__(kThreads) accumulate_kernel(const double* __restrict__ f,
                                                              const double* __restrict__ factor,
                                                              const int32_t* __restrict__ bin, uint64_t n, int dims,
                                                              int bins, double* __restrict__ partial,
                                                              int32_t* __restrict__ counts)
{
    extern __shared__ double hsm[];  // [warps][dims*bins]
    __shared__ double red[2][kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < kWarps * dims * bins; k += blockDim.x) hsm[k] = 0.0;
    __syncthreads();
    double* myhist = hsm + warp * dims * bins;
    const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t begin = (uint64_t)blockIdx.x * chunk;
    const uint64_t end = begin + chunk < n ? begin + chunk : n;
    double s = 0.0, s2 = 0.0;
    for (uint64_t base = begin; base < end; base += kThreads) {
        const uint64_t i = base + threadIdx.x;
        const bool on = i < end;
        const double w = on ? f[i] * factor[i] : 0.0;
        s += w;
        s2 += w * w;
        const unsigned mask = __ballot_sync(0xffffffffu, on);
        if (on) {
            const double aw = ::fabs(w);
            for (int d = 0; d < dims; ++d) {
                const int key = d * bins + bin[i * dims + d];
                const unsigned peers = __match_any_sync(mask, key);
                const int rank = __popc(peers & ((1u << lane) - 1u));
                const int last = __reduce_max_sync(mask, rank);
                for (int k = 0; k <= last; ++k) {
                    if (rank == k) myhist[key] += aw;
                    __syncwarp(mask);
                }
                atomicAdd(&counts[key], 1);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
        red[0][warp] = s;
        red[1][warp] = s2;
    }
    __syncthreads();
    double* out = partial + (size_t)blockIdx.x * (2 + dims * bins);
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < kWarps; ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        out[0] = a;
        out[1] = b;
    }
    for (int k = threadIdx.x; k < dims * bins; k += blockDim.x) {
        double h = 0.0;
        for (int w = 0; w < kWarps; ++w) h += hsm[w * dims * bins + k];
        out[2 + k] = h;
    }
}

__global__ void add_kernel(double* __restrict__ round, const double* __restrict__ batch, int keys)
{
    for (int k = threadIdx.x; k < keys; k += blockDim.x) round[k] += batch[k];
}

__global__ void end_round_kernel(double* state, int dims, int bins, uint64_t samples, double* __restrict__ round,
                                 int32_t* __restrict__ counts, int warmup, int min_iterations, double epsrel,
                                 double epsabs)
{
    extern __shared__ double fsm[];
    double* smooth = fsm;
    double* cum = smooth + dims * bins;
    double* next = cum + dims * (bins + 1);
    double* sc = state + dims * (bins + 1);
    rebin(state, round + 2, counts, dims, bins, smooth, cum, next);
    __syncthreads();
    if (threadIdx.x == 0) {
        sc[kStEvals] += (double)samples;
        if (!warmup) combine(sc, round[0], round[1], (double)samples, min_iterations, epsrel, epsabs);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < dims * bins; k += blockDim.x) counts[k] = 0;
    for (int k = threadIdx.x; k < 2 + dims * bins; k += blockDim.x) round[k] = 0.0;
}

bool check_shape(int dims, int bins, std::string& why)
{
    if (dims < 1 || dims > kMaxDims) { why = "dims must be 1..8"; return false; }
    if (bins < 2 || bins > 256) { why = "bins must be 2..256"; return false; }
    return true;
}

}  // namespace

}  // namespace nlo

using namespace nlo;

extern "C" {

size_t nlo_vegas_state_doubles(int32_t dims, int32_t bins)
{
    std::string why;
    return check_shape(dims, bins, why) ? (size_t)dims * (bins + 1) + kStSlots : 0;
}

size_t nlo_vegas_workspace_bytes(int32_t dims, int32_t bins)
{
    std::string why;
    if (!check_shape(dims, bins, why)) return 0;
    const size_t keys = keys_of(dims, bins);
    return sizeof(double) * keys * (kBlocks + 2) + sizeof(int32_t) * (size_t)dims * bins;
}

int nlo_vegas_begin(int32_t dims, int32_t bins, int32_t keep_edges, double* state, void* workspace,
                    size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!check_shape(dims, bins, why)) return set_last_error(NLO_ERR_INVALID, why.c_str());
    if (!state) return set_last_error(NLO_ERR_INVALID, "NULL buffer");
    if (!workspace || workspace_bytes < nlo_vegas_workspace_bytes(dims, bins))
        return set_last_error(NLO_ERR_WORKSPACE, "workspace too small for nlo_vegas_begin");
    const GenericBuffers b = carve_generic(workspace, dims, bins);
    begin_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(state, dims, bins, keep_edges ? 1 : 0, b.round, b.counts);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NLO_OK : set_last_error(NLO_ERR_CUDA, cudaGetErrorString(e));
}

int nlo_vegas_sample(const nlo_sobol_dirs* dirs, int64_t offset, int64_t n, int32_t dims, int32_t bins,
                     const double* state, const double* lower, const double* width, double* x, double* factor,
                     int32_t* bin, void* stream)
{
    std::string why;
    if (!check_shape(dims, bins, why)) return set_last_error(NLO_ERR_INVALID, why.c_str());
    if (!check_dirs(dirs, dims, why)) return set_last_error(NLO_ERR_INVALID, why.c_str());
    if (offset < 0 || n < 0 || offset + n > (int64_t(1) << 30))
        return set_last_error(NLO_ERR_INVALID, "Sobol index range exceeds 2^30");
    if (!state || !lower || !width || (n > 0 && (!x || !factor || !bin)))
        return set_last_error(NLO_ERR_INVALID, "NULL buffer");
    if (n == 0) return NLO_OK;
    BoxArg box;
    box.volume = 1.0;
    for (int d = 0; d < kMaxDims; ++d) {
        box.lower[d] = d < dims ? lower[d] : 0.0;
        box.width[d] = d < dims ? width[d] : 0.0;
        if (d < dims) box.volume *= width[d];
    }
    const size_t smem = sizeof(double) * (size_t)dims * (bins + 1);
    uint64_t blocks = ((uint64_t)n + 255) / 256;
    blocks = blocks > 4096 ? 4096 : blocks;
    sample_kernel<<<(unsigned)blocks, 256, smem, (cudaStream_t)stream>>>(to_arg(dirs), (uint64_t)offset, (uint64_t)n,
                                                                         dims, bins, state, box, x, factor, bin);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NLO_OK : set_last_error(NLO_ERR_CUDA, cudaGetErrorString(e));
}

int nlo_vegas_accumulate(const double* f, const double* factor, const int32_t* bin, int64_t n, int32_t dims,
                         int32_t bins, void* workspace, size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!check_shape(dims, bins, why)) return set_last_error(NLO_ERR_INVALID, why.c_str());
    if (n < 0) return set_last_error(NLO_ERR_INVALID, "n must be non-negative");
    if (n > 0 && (!f || !factor || !bin)) return set_last_error(NLO_ERR_INVALID, "NULL buffer");
    if (!workspace || workspace_bytes < nlo_vegas_workspace_bytes(dims, bins))
        return set_last_error(NLO_ERR_WORKSPACE, "workspace too small for nlo_vegas_accumulate");
    if (n == 0) return NLO_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const GenericBuffers b = carve_generic(workspace, dims, bins);
    const int keys = (int)keys_of(dims, bins);
    const size_t smem = sizeof(double) * kWarps * (size_t)dims * bins;
    cudaError_t e = raise_dynamic_smem((const void*)accumulate_kernel, smem);
    if (e == cudaSuccess) {
        accumulate_kernel<<<kBlocks, kThreads, smem, s>>>(f, factor, bin, (uint64_t)n, dims, bins, b.partial,
                                                          b.counts);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = vegas_launch_reduce(b.partial, keys, kBlocks, 1, b.batch, s);
    if (e == cudaSuccess) {
        add_kernel<<<1, 256, 0, s>>>(b.round, b.batch, keys);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? NLO_OK : set_last_error(NLO_ERR_CUDA, cudaGetErrorString(e));
}

int nlo_vegas_end_round(int32_t dims, int32_t bins, double* state, int64_t samples, int32_t warmup,
                        int32_t min_iterations, double epsrel, double epsabs, void* workspace, size_t workspace_bytes,
                        void* stream)
{
    std::string why;
    if (!check_shape(dims, bins, why)) return set_last_error(NLO_ERR_INVALID, why.c_str());
    if (!state) return set_last_error(NLO_ERR_INVALID, "NULL buffer");
    if (samples < 2) return set_last_error(NLO_ERR_INVALID, "a Vegas round needs at least two samples");
    if (!workspace || workspace_bytes < nlo_vegas_workspace_bytes(dims, bins))
        return set_last_error(NLO_ERR_WORKSPACE, "workspace too small for nlo_vegas_end_round");
    const GenericBuffers b = carve_generic(workspace, dims, bins);
    const size_t smem = sizeof(double) * ((size_t)dims * bins + 2 * (size_t)dims * (bins + 1));
    cudaError_t e = raise_dynamic_smem((const void*)end_round_kernel, smem);
    if (e == cudaSuccess) {
        end_round_kernel<<<1, 128, smem, (cudaStream_t)stream>>>(state, dims, bins, (uint64_t)samples, b.round,
                                                                 b.counts, warmup ? 1 : 0, min_iterations, epsrel,
                                                                 epsabs);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? NLO_OK : set_last_error(NLO_ERR_CUDA, cudaGetErrorString(e));
}

}  // extern "C"
