// K2 + Kf by Vegas: the reference's default integrator for the NLO part of the BK
// right-hand side (rapidity_derivative_nlo with IntegrationMethod.VEGAS,
// bk/derivatives.py:389-421 -- 32 bins, a warm-up of max(2, MCINTPOINTS/5) samples, at
// least 2 and at most 4 iterations, epsrel 0.2 -- driving vegas(), numerics/integration.py:
// 120-589), with each parent's importance grid carried from one right-hand side to the next
// and refreshed by a shortened warm-up (VEGAS_REUSE_GRID, VEGAS_REUSE_WARMUP_FRACTION; the
// per-parent vegas_states of bk/evolution.py:85-100 and 354-424).
//
// Every active parent is one integral with its own grid; all of them run in the same
// launches.  A round (the warm-up, or one iteration) is three launches: the round kernel
// (grid: CTAs per parent x grid points) maps scrambled Sobol points through the parent's
// grid, evaluates the full integrand and leaves per-CTA sums of w, w^2, w_K2, w_Kf and the
// |w| histograms; a fixed-order reduction over the CTAs; and a finalize CTA per parent that
// re-bins the grid and folds the iteration into the inverse-variance combination
// (vegas_common.cuh, the code the DIS terms use).  Converged parents skip the remaining
// rounds, so the host enqueues every round without synchronising.
//
// Samples: the Sobol points of `dirs`, indices 0, 1, ... across the rounds of one
// right-hand side (the warm-up first); every parent and every right-hand side starts again
// at index 0, as the reference restarts its generator from the same seed in every vegas()
// call.  A coordinate u gives the bin floor(u bins) and the fraction u bins - bin.
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "k2kf_integrand.cuh"
#include "sobol.cuh"
#include "vegas_common.cuh"

namespace nlo {

namespace {

using namespace k2;
using namespace vegas;

constexpr int kDims = 4;
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// BK slots after the generic ones of vegas_common.cuh (all < kStSlots)
enum BkSlot {
    kBkHasGrid = 9,   // the grid was adapted by an earlier right-hand side (persistent)
    kBkWarmup = 10,   // warm-up samples of this right-hand side
    kBkOffset = 11,   // Sobol index of the next round
    kBkActive = 12,   // the parent is integrated in this right-hand side
    kBkCompK2 = 13,   // sum over iterations of weight x K2 estimate
    kBkCompKf = 14,   // sum over iterations of weight x Kf estimate
};

// Per-parent accumulators of the replica refinement: [selected, sum of values, sum of error^2].
constexpr int kRepStride = 3;

__device__ __forceinline__ bool parent_active(const double* N, int i, int shard, int shards)
{
    return i > 0 && N[i] <= 0.99999 && i % shards == shard;
}

// Per parent: mark whether it is integrated, reset the per-call sums, and either start a
// uniform grid with the full warm-up or keep the stored grid with the reuse warm-up.
// select (replica rounds): the parents to integrate are those with select[i * kRepStride] != 0.
__global__ void begin_kernel(const double* __restrict__ N, int points, int shard, int shards, double* state,
                             int stride, int bins, int reuse, uint64_t warmup, uint64_t reuse_warmup,
                             int32_t* __restrict__ counts, const double* __restrict__ select)
{
    const int i = blockIdx.x;
    double* st = state + (size_t)i * stride;
    double* sc = st + kDims * (bins + 1);
    const bool on = select ? select[(size_t)i * kRepStride] != 0.0 : parent_active(N, i, shard, shards);
    __syncthreads();
    const bool fresh = !reuse || sc[kBkHasGrid] == 0.0;
    if (on) {
        for (int k = threadIdx.x; k < kDims * bins; k += blockDim.x) counts[(size_t)i * kDims * bins + k] = 0;
        if (fresh)
            for (int k = threadIdx.x; k < kDims * (bins + 1); k += blockDim.x) {
                const int b = k % (bins + 1);
                st[k] = b == bins ? 1.0 : (double)b / bins;
            }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (on) {
            for (int k = 0; k <= kStLastVariance; ++k) sc[k] = 0.0;
            sc[kBkCompK2] = 0.0;
            sc[kBkCompKf] = 0.0;
            sc[kBkWarmup] = (double)(fresh ? warmup : reuse_warmup);
            sc[kBkOffset] = 0.0;
        }
        sc[kBkActive] = on ? 1.0 : 0.0;
    }
}

// Samples of parent slot `sc` in this round (0: skip the parent).
__device__ __forceinline__ uint64_t round_samples(const double* sc, int warmup, uint64_t samples)
{
    if (sc[kBkActive] == 0.0 || sc[kStConverged] != 0.0) return 0;
    return warmup ? (uint64_t)sc[kBkWarmup] : samples;
}

template <typename T, bool SYM>
__global__ void __launch_bounds__(kThreads) round_kernel(Phys<T> ph, K2Box<T> box, SobolDirsArg dirs,
                                                         const double* __restrict__ r_grid, int n,
                                                         const double* __restrict__ spline, const double* state,
                                                         int stride, int bins, int warmup, uint64_t samples,
                                                         int blocks_per_job, double* __restrict__ partial,
                                                         int32_t* __restrict__ counts)
{
    const int job = blockIdx.y;
    const double* st = state + (size_t)job * stride;
    const double* sc = st + kDims * (bins + 1);
    const uint64_t total = round_samples(sc, warmup, samples);
    if (total == 0) return;  // uniform per CTA

    extern __shared__ __align__(16) unsigned char vsm[];
    double* edges = reinterpret_cast<double*>(vsm);                       // [4][bins+1]
    double* whist = edges + kDims * (bins + 1);                           // [warps][4*bins]
    int32_t* cnt = reinterpret_cast<int32_t*>(whist + kWarps * kDims * bins);  // [4*bins]
    T* xs = reinterpret_cast<T*>(cnt + kDims * bins + 4);                 // [n] (16-byte aligned)
    T* cs = xs + ((n + 3) & ~3);                                          // [n-1][4] log S block
    __shared__ uint32_t sst[kDims][30];
    __shared__ uint32_t ssh[kDims];
    __shared__ double red[4][kWarps];

    const double* src_coef = spline + n + 4 * (size_t)(n - 1);
    for (int k = threadIdx.x; k < kDims * (bins + 1); k += blockDim.x) edges[k] = st[k];
    for (int k = threadIdx.x; k < kWarps * kDims * bins; k += blockDim.x) whist[k] = 0.0;
    for (int k = threadIdx.x; k < kDims * bins; k += blockDim.x) cnt[k] = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = (T)spline[i];
    for (int i = threadIdx.x; i < 4 * (n - 1); i += blockDim.x) cs[i] = (T)src_coef[i];
    for (int k = threadIdx.x; k < kDims * 30; k += blockDim.x) sst[k / 30][k % 30] = dirs.state[k / 30][k % 30];
    if (threadIdx.x < kDims) ssh[threadIdx.x] = dirs.shift[threadIdx.x];
    __syncthreads();

    SplineView<T> s;
    s.x = xs;
    s.coef = cs;
    s.n = n;
    s.x0 = xs[0];
    s.inv_h = (T)((double)(n - 1) / (spline[n - 1] - spline[0]));
    K2Parent<T> P;
    {
        const double r = r_grid[job];
        P.r = (T)r;
        P.r2 = P.r * P.r;
        P.lr = (T)log(r);
        P.two_r = (T)2 * P.r;
        P.alpha_r = alpha_of_log(P.lr, ph);
    }
    const double lower[kDims] = {(double)box.lower[0], (double)box.lower[1], (double)box.lower[2],
                                 (double)box.lower[3]};
    const double width[kDims] = {(double)box.width[0], (double)box.width[1], (double)box.width[2],
                                 (double)box.width[3]};

    const uint64_t offset = (uint64_t)sc[kBkOffset];
    const uint64_t chunk = (total + blocks_per_job - 1) / blocks_per_job;
    const uint64_t begin = (uint64_t)blockIdx.x * chunk;
    const uint64_t end = begin + chunk < total ? begin + chunk : total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* myhist = whist + warp * kDims * bins;
    const double fb = (double)bins;
    double sw = 0.0, sw2 = 0.0, sk2 = 0.0, skf = 0.0;
    for (uint64_t base = begin; base < end; base += kThreads) {
        const uint64_t i = base + threadIdx.x;
        const bool on = i < end;
        int bin[kDims];
        double w = 0.0, wk2 = 0.0, wkf = 0.0;
        if (on) {
            const uint64_t index = offset + i;
            T x[kDims];
            double inv_density = 1.0;
#pragma unroll
            for (int d = 0; d < kDims; ++d) {
                const double u = sobol_unit<double>(sobol_bits(sst[d], ssh[d], index), index);
                const double scaled = u * fb;
                int b = (int)floor(scaled);
                b = b > bins - 1 ? bins - 1 : b;
                const double frac = scaled - b;
                const double left = edges[d * (bins + 1) + b];
                const double bw = edges[d * (bins + 1) + b + 1] - left;
                x[d] = (T)(lower[d] + width[d] * (left + bw * frac));
                inv_density *= fb * bw;
                bin[d] = b;
            }
            T rec[kRecLen];
            k2_prepare_x<T>(s, box, x, true, rec);
            T k2w, kfw;
            k2_point<T, SYM>(s, ph, P, rec, k2w, kfw);
            wk2 = (double)k2w * inv_density;
            wkf = (double)kfw * inv_density;
            w = ((double)k2w + (double)kfw) * inv_density;
        }
        sw += w;
        sw2 += w * w;
        sk2 += wk2;
        skf += wkf;
        // deterministic warp histogram: lanes that share a bin add in lane order
        const unsigned mask = __ballot_sync(0xffffffffu, on);
        if (on) {
            const double aw = ::fabs(w);
#pragma unroll
            for (int d = 0; d < kDims; ++d) {
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
    for (int o = 16; o > 0; o >>= 1) {
        sw += __shfl_down_sync(0xffffffffu, sw, o);
        sw2 += __shfl_down_sync(0xffffffffu, sw2, o);
        sk2 += __shfl_down_sync(0xffffffffu, sk2, o);
        skf += __shfl_down_sync(0xffffffffu, skf, o);
    }
    if (lane == 0) {
        red[0][warp] = sw;
        red[1][warp] = sw2;
        red[2][warp] = sk2;
        red[3][warp] = skf;
    }
    __syncthreads();
    // partial row: [sum w, sum w^2, hist[4][bins], sum w_K2, sum w_Kf]
    const int keys = 4 + kDims * bins;
    double* out = partial + ((size_t)job * blocks_per_job + blockIdx.x) * keys;
    if (threadIdx.x == 0) {
        double a[4] = {0.0, 0.0, 0.0, 0.0};
        for (int w = 0; w < kWarps; ++w)
            for (int q = 0; q < 4; ++q) a[q] += red[q][w];
        out[0] = a[0];
        out[1] = a[1];
        out[2 + kDims * bins] = a[2];
        out[3 + kDims * bins] = a[3];
    }
    int32_t* cout = counts + (size_t)job * kDims * bins;
    for (int k = threadIdx.x; k < kDims * bins; k += blockDim.x) {
        double h = 0.0;
        for (int w = 0; w < kWarps; ++w) h += whist[w * kDims * bins + k];
        out[2 + k] = h;
        if (cnt[k]) atomicAdd(&cout[k], cnt[k]);
    }
}

// Per parent: re-bin the grid from the round's histogram and, for an iteration, fold its
// estimate into the weighted combination (value, error, convergence) and the K2 / Kf
// components; then advance the Sobol offset.
__global__ void finalize_kernel(double* state, int stride, int bins, int warmup, uint64_t samples,
                                const double* __restrict__ reduced, int32_t* __restrict__ counts, int min_iterations,
                                double epsrel, double epsabs)
{
    extern __shared__ double fsm[];
    double* smooth = fsm;                    // [4*bins]
    double* cum = smooth + kDims * bins;     // [4*(bins+1)]
    double* next = cum + kDims * (bins + 1); // [4*(bins+1)]
    const int job = blockIdx.x;
    double* st = state + (size_t)job * stride;
    double* sc = st + kDims * (bins + 1);
    const uint64_t n_round = round_samples(sc, warmup, samples);
    if (n_round == 0) return;
    const int keys = 4 + kDims * bins;
    const double* red = reduced + (size_t)job * keys;
    int32_t* c = counts + (size_t)job * kDims * bins;
    rebin(st, red + 2, c, kDims, bins, smooth, cum, next);
    __syncthreads();
    for (int k = threadIdx.x; k < kDims * bins; k += blockDim.x) c[k] = 0;
    if (threadIdx.x == 0) {
        const double n = (double)n_round;
        sc[kStEvals] += n;
        if (!warmup) {
            const double weight = combine(sc, red[0], red[1], n, min_iterations, epsrel, epsabs);
            sc[kBkCompK2] += weight * (red[2 + kDims * bins] / n);
            sc[kBkCompKf] += weight * (red[3 + kDims * bins] / n);
        }
        sc[kBkOffset] += n;
        sc[kBkHasGrid] = 1.0;
    }
}

// The right-hand side's K2+Kf per parent in the layout of nlo_bk_k2kf's sums: [value, 0,
// error^2] (assembled with the factor 1), zeros for parents not integrated.
__global__ void end_kernel(const double* state, int stride, int bins, int points, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= points) return;
    const double* sc = state + (size_t)i * stride + kDims * (bins + 1);
    const bool on = sc[kBkActive] != 0.0;
    out[3 * i + 0] = on ? sc[kStValue] : 0.0;
    out[3 * i + 1] = 0.0;
    out[3 * i + 2] = on ? sc[kStError] * sc[kStError] : 0.0;
}

// Replica refinement of bk/evolution.py:411-456 (the reference's CUDA mixed evolution with
// per-parent grids): a parent whose K1 and combined K2, Kf estimates cancel strongly,
// (|K1| + |K2| + |Kf|) / max(|K1 + K2 + Kf|, 0.05 (|K1| + |K2| + |Kf|)) >= 4, or whose
// amplitude exceeds 0.9, gets `replicas` more Vegas integrals on fresh grids with the seeds
// seed + 1000 k, and its K2+Kf becomes the mean of all of them, with the error
// sqrt(sum error^2) / (replicas + 1).  The parent's own grid is kept.
__global__ void replica_select_kernel(const double* __restrict__ N, const double* __restrict__ k1, int points,
                                      const double* __restrict__ state, int stride, int bins,
                                      double* __restrict__ acc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= points) return;
    const double* sc = state + (size_t)i * stride + kDims * (bins + 1);
    double* a = acc + (size_t)i * kRepStride;
    a[0] = 0.0;
    if (sc[kBkActive] == 0.0 || !(sc[kStSumWeights] > 0.0)) return;
    const double c2 = sc[kBkCompK2] / sc[kStSumWeights];
    const double cf = sc[kBkCompKf] / sc[kStSumWeights];
    const double scale = ::fabs(k1[i]) + ::fabs(c2) + ::fabs(cf);
    const double net = ::fabs(k1[i] + c2 + cf);
    const double condition = scale / (net > 0.05 * scale ? net : 0.05 * scale);
    if (condition >= 4.0 || N[i] > 0.9) {
        a[0] = 1.0;
        a[1] = sc[kStValue];
        a[2] = sc[kStError] * sc[kStError];
    }
}

__global__ void replica_add_kernel(const double* __restrict__ state, int stride, int bins, int points,
                                   double* __restrict__ acc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= points) return;
    double* a = acc + (size_t)i * kRepStride;
    if (a[0] == 0.0) return;
    const double* sc = state + (size_t)i * stride + kDims * (bins + 1);
    a[1] += sc[kStValue];
    a[2] += sc[kStError] * sc[kStError];
}

__global__ void replica_end_kernel(const double* __restrict__ acc, int points, int replicas, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= points) return;
    const double* a = acc + (size_t)i * kRepStride;
    if (a[0] == 0.0) return;
    const double m = (double)(replicas + 1);
    out[3 * i + 0] = a[1] / m;
    out[3 * i + 2] = a[2] / (m * m);
}

template <typename T, bool SYM>
cudaError_t launch_round(const nlo_bk_params& p, const double* r, int points, const double* spline,
                         const SobolDirsArg& dirs, const nlo_bk_box& box, const BkVegasCall& call, int warmup,
                         cudaStream_t stream)
{
    const int bins = call.options.bins;
    const size_t smem = sizeof(double) * (kDims * (bins + 1) + kWarps * kDims * bins) +
                        sizeof(int32_t) * (kDims * bins + 4) + sizeof(T) * (((points + 3) & ~3) + 4 * (points - 1));
    auto kern = round_kernel<T, SYM>;
    cudaError_t e = raise_dynamic_smem((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    K2Box<T> kb;
    for (int d = 0; d < 4; ++d) {
        kb.lower[d] = (T)box.lower[d];
        kb.width[d] = (T)box.width[d];
    }
    const double volume = box.width[0] * box.width[1] * box.width[2] * box.width[3];
    kb.cpt_scale = (T)(volume * p.nc * p.nc / (8.0 * kPi * kPi * kPi * kPi));
    dim3 grid((unsigned)call.blocks_per_job, (unsigned)points);
    kern<<<grid, kThreads, smem, stream>>>(make_phys<T>(p), kb, dirs, r, points, spline, call.state,
                                           call.stride, bins, warmup, (uint64_t)call.options.samples_per_iteration,
                                           call.blocks_per_job, call.partial, call.counts);
    return cudaGetLastError();
}

// The warm-up round (when `with_warmup`) and the iterations of one Vegas call over the
// parents that `call.state` marks active.
cudaError_t run_rounds(const nlo_bk_params& p, const double* r, int points, const double* spline,
                       const SobolDirsArg& dirs, const nlo_bk_box& box, const BkVegasCall& call, bool with_warmup,
                       cudaStream_t stream)
{
    const nlo_bk_vegas_options& o = call.options;
    const bool fp64 = p.precision == NLO_PRECISION_FP64;
    const bool sym = p.symmetrize != 0;
    const int keys = 4 + kDims * o.bins;
    const size_t fsmem = sizeof(double) * (kDims * o.bins + 2 * kDims * (o.bins + 1));
    cudaError_t e = raise_dynamic_smem((const void*)finalize_kernel, fsmem);
    if (e != cudaSuccess) return e;
    const int rounds = o.max_iterations + (with_warmup ? 1 : 0);
    for (int k = 0; k < rounds; ++k) {
        const int is_warmup = with_warmup && k == 0;
        if (fp64)
            e = sym ? launch_round<double, true>(p, r, points, spline, dirs, box, call, is_warmup, stream)
                    : launch_round<double, false>(p, r, points, spline, dirs, box, call, is_warmup, stream);
        else
            e = sym ? launch_round<float, true>(p, r, points, spline, dirs, box, call, is_warmup, stream)
                    : launch_round<float, false>(p, r, points, spline, dirs, box, call, is_warmup, stream);
        if (e != cudaSuccess) return e;
        if ((e = vegas_launch_reduce(call.partial, keys, call.blocks_per_job, points, call.reduced, stream)) !=
            cudaSuccess)
            return e;
        finalize_kernel<<<points, 128, fsmem, stream>>>(call.state, call.stride, o.bins, is_warmup,
                                                        (uint64_t)o.samples_per_iteration, call.reduced, call.counts,
                                                        o.min_iterations, o.epsrel, o.epsabs);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

size_t bk_vegas_state_doubles(int bins) { return (size_t)kDims * (bins + 1) + kStSlots; }

int bk_vegas_blocks_per_job(int points)
{
    int device = 0, sms = 148;
    if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    // about two waves of 256-thread CTAs at six per SM over all grid points
    const int target = 2 * 6 * (sms > 0 ? sms : 148);
    int b = (target + points - 1) / points;
    return b < 1 ? 1 : (b > 64 ? 64 : b);
}

size_t bk_vegas_scratch_bytes(int points, int bins)
{
    const size_t keys = 4 + (size_t)kDims * bins;
    const size_t blocks = (size_t)bk_vegas_blocks_per_job(points);
    // round partials and sums, bin counts, then the replica grids and accumulators
    return sizeof(double) * keys * (size_t)points * (blocks + 1) + sizeof(int32_t) * (size_t)kDims * bins * points +
           256 + sizeof(double) * (bk_vegas_state_doubles(bins) + kRepStride) * (size_t)points + 256;
}

BkVegasCall bk_vegas_carve(void* scratch, int points, const nlo_bk_vegas_options& options, double* state)
{
    BkVegasCall c;
    c.options = options;
    c.state = state;
    c.stride = (int)bk_vegas_state_doubles(options.bins);
    c.blocks_per_job = bk_vegas_blocks_per_job(points);
    const size_t keys = 4 + (size_t)kDims * options.bins;
    char* base = static_cast<char*>(scratch);
    c.partial = reinterpret_cast<double*>(base);
    c.reduced = c.partial + keys * (size_t)points * (size_t)c.blocks_per_job;
    c.counts = reinterpret_cast<int32_t*>(c.reduced + keys * (size_t)points);
    const size_t after = reinterpret_cast<size_t>(c.counts + (size_t)kDims * options.bins * points);
    c.replica_state = reinterpret_cast<double*>((after + 255) & ~(size_t)255);
    c.replica_acc = c.replica_state + bk_vegas_state_doubles(options.bins) * (size_t)points;
    return c;
}

cudaError_t launch_k2kf_vegas(const nlo_bk_params& p, const double* r, const double* N, int points,
                              const double* spline, int shard, int shards, const SobolDirsArg& dirs,
                              const nlo_bk_box& box, const BkVegasCall& call, double* out, cudaStream_t stream)
{
    const nlo_bk_vegas_options& o = call.options;
    const uint64_t warmup = (uint64_t)o.warmup_samples;
    // numerics/integration.py:207-213: a reused grid is refreshed by max(2, warmup x fraction)
    // samples, or none when the warm-up or the fraction is zero
    uint64_t reuse_warmup = 0;
    if (warmup > 0 && o.reuse_warmup_fraction > 0.0) {
        reuse_warmup = (uint64_t)((double)warmup * o.reuse_warmup_fraction);
        if (reuse_warmup < 2) reuse_warmup = 2;
    }
    begin_kernel<<<points, 64, 0, stream>>>(N, points, shard, shards, call.state, call.stride, o.bins,
                                             o.reuse_grid ? 1 : 0, warmup, reuse_warmup, call.counts, nullptr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = run_rounds(p, r, points, spline, dirs, box, call, warmup > 0 || reuse_warmup > 0, stream)) !=
        cudaSuccess)
        return e;
    end_kernel<<<(points + 255) / 256, 256, 0, stream>>>(call.state, call.stride, o.bins, points, out);
    return cudaGetLastError();
}

cudaError_t launch_k2kf_vegas_refine(const nlo_bk_params& p, const double* r, const double* N, int points,
                                     const double* spline, const nlo_bk_box& box, const BkVegasCall& call,
                                     const double* k1, double* out, cudaStream_t stream)
{
    const nlo_bk_vegas_options& o = call.options;
    if (o.replicas <= 0) return cudaSuccess;
    const int threads = 128, blocks = (points + threads - 1) / threads;
    replica_select_kernel<<<blocks, threads, 0, stream>>>(N, k1, points, call.state, call.stride, o.bins,
                                                          call.replica_acc);
    cudaError_t e = cudaGetLastError();
    // each replica: a fresh grid with the full warm-up (the reference's new VegasState)
    BkVegasCall rep = call;
    rep.state = call.replica_state;
    const uint64_t warmup = (uint64_t)o.warmup_samples;
    for (int k = 0; k < o.replicas && e == cudaSuccess; ++k) {
        begin_kernel<<<points, 64, 0, stream>>>(N, points, 0, 1, rep.state, rep.stride, o.bins, 0, warmup, 0,
                                                 rep.counts, call.replica_acc);
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        if ((e = run_rounds(p, r, points, spline, call.replica_dirs[k], box, rep, warmup > 0, stream)) != cudaSuccess)
            break;
        replica_add_kernel<<<blocks, threads, 0, stream>>>(rep.state, rep.stride, o.bins, points, call.replica_acc);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    replica_end_kernel<<<blocks, threads, 0, stream>>>(call.replica_acc, points, o.replicas, out);
    return cudaGetLastError();
}

}  // namespace nlo
