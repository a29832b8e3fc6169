// Fixed-Sobol qqbar-g integration (dis/fixed_sobol.py:66-368, endpoint map
// custom_kernels/dis/sampling/kernel.cu:15-84) on the device.
//
// One request = one (Q^2, x_Bj, quark, polarisation).  Training: for each of R rounds,
// Sobol points of seed + r are mapped through the current grid, the gluon plane is split by
// the nearer dipole end (two weighted evaluations per point), I1, I2 and I3 are evaluated
// together, the per-point score sum_k w_k |I_k| / mean|I_k| fills the bin histograms and
// the grid is re-binned exactly like a Vegas round.  Estimation: each replicate (seed
// 10000 + j) is mapped through the frozen grid and its three means are written out; the
// host forms the mean and the replicate standard error.  No host synchronisation inside.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dis_internal.h"
#include "dis_terms.cuh"
#include "sobol.cuh"

namespace nlo {
namespace dis {

constexpr int kFixedDims = 5;
constexpr int kFixedThreads = 256;

struct FixedGeom {
    double maxr;
    int bins;
    int fold;
};

// map_importance_grid (dis/fixed_sobol.py:100-112) and paired_endpoint_inputs (:115-158)
__device__ __forceinline__ void endpoint_map(const double* __restrict__ edges, const FixedGeom& g, const float* u,
                                             double first[kFixedDims], double second[kFixedDims], double& fw,
                                             double& sw, int bin[kFixedDims])
{
    double src[kFixedDims];
    double inv = 1.0;
    const double fb = (double)g.bins;
#pragma unroll
    for (int d = 0; d < kFixedDims; ++d) {
        const double scaled = (double)u[d] * fb;
        int b = (int)floor(scaled);
        b = b > g.bins - 1 ? g.bins - 1 : b;
        const double frac = scaled - b;
        const double left = edges[d * (g.bins + 1) + b];
        const double width = edges[d * (g.bins + 1) + b + 1] - left;
        src[d] = left + width * frac;
        inv *= fb * width;
        bin[d] = b;
        first[d] = src[d];
        second[d] = src[d];
    }
    const double parent = g.maxr * src[2];
    const double radial = src[3];
    const double af = g.fold ? 0.5 * src[4] : src[4];
    const double angle = 2.0 * kPi * af;
    const double c = ::cos(angle), s = ::sin(angle);
    const double closer = c > 0.0 ? parent / (2.0 * (c > 2.2250738585072014e-308 ? c : 2.2250738585072014e-308))
                                  : CUDART_INF;
    const double first_limit = g.maxr < closer ? g.maxr : closer;
    first[3] = radial * first_limit / g.maxr;
    first[4] = af;
    fw = inv * first_limit / g.maxr;
    const double disk_arg = g.maxr * g.maxr - parent * parent * s * s;
    const double disk = parent * c + ::sqrt(disk_arg > 0.0 ? disk_arg : 0.0);
    double second_limit = disk < closer ? disk : closer;
    second_limit = second_limit > 0.0 ? second_limit : 0.0;
    const double sr = radial * second_limit;
    const double gx = parent - sr * c, gy = sr * s;
    const double gr = ::sqrt(gx * gx + gy * gy);
    double ga = ::atan2(gy, gx);
    if (ga < 0.0) ga += 2.0 * kPi;
    second[3] = gr / g.maxr;
    second[4] = ga / (2.0 * kPi);
    sw = inv * sr * second_limit / ((gr > 2.2250738585072014e-308 ? gr : 2.2250738585072014e-308) * g.maxr);
}

// TRAIN = true: per-point weighted (I1, I2, I3) and bins to global memory.
// TRAIN = false: per-CTA sums of the weighted values (fixed order).
template <typename T, bool TRAIN>
__global__ void __launch_bounds__(kFixedThreads, 3) fixed_triple_kernel(
    const DisArgs<T> args, const InnerRule rule, const SobolDirsArg* __restrict__ dirs, int dir_base, uint64_t n,
    const double* __restrict__ edges, FixedGeom g, double* __restrict__ wout, uint8_t* __restrict__ bout,
    double* __restrict__ partial)
{
    __shared__ __align__(16) unsigned char raw[sizeof(DisArgs<T>)];
    DisArgs<T>& a = *reinterpret_cast<DisArgs<T>*>(raw);
    __shared__ uint32_t sst[kFixedDims][30];
    __shared__ uint32_t ssh[kFixedDims];
    __shared__ double red[3][kFixedThreads / 32];
    if (threadIdx.x == 0) a = args;
    const SobolDirsArg& sd = dirs[dir_base + blockIdx.y];  // replicates: one per grid row
    for (int k = threadIdx.x; k < kFixedDims * 30; k += blockDim.x) sst[k / 30][k % 30] = sd.state[k / 30][k % 30];
    if (threadIdx.x < kFixedDims) ssh[threadIdx.x] = sd.shift[threadIdx.x];
    __syncthreads();
    // Two lanes per sample: the even lane evaluates the first endpoint, the odd lane the
    // second, and the even lane forms the sample's weight from its partner's values by the
    // same expression as one lane would.  The loop runs over whole warps (the stride is a
    // multiple of 32) so that every lane reaches the exchange.
    double acc[3] = {0.0, 0.0, 0.0};
    const uint64_t lanes = 2 * n;
    const uint64_t span = (lanes + 31) & ~(uint64_t)31;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < span; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = t >> 1;
        const bool odd = (t & 1) != 0;
        const bool valid = t < lanes;
        double fw = 0.0, sw = 0.0;
        int bin[kFixedDims];
        T v[3] = {(T)0, (T)0, (T)0};
        if (valid) {
            float u[kFixedDims];
#pragma unroll
            for (int d = 0; d < kFixedDims; ++d) u[d] = sobol_unit<float>(sobol_bits(sst[d], ssh[d], i), i);
            double first[kFixedDims], second[kFixedDims];
            endpoint_map(edges, g, u, first, second, fw, sw, bin);
            qg_triple(a, odd ? second : first, rule, v);
        }
        T v2[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) v2[k] = __shfl_xor_sync(0xffffffffu, v[k], 1);
        if (valid && !odd) {
            double w[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) w[k] = (double)v[k] * fw + (double)v2[k] * sw;
            if constexpr (TRAIN) {
#pragma unroll
                for (int k = 0; k < 3; ++k) wout[i * 3 + k] = w[k];
#pragma unroll
                for (int d = 0; d < kFixedDims; ++d) bout[i * kFixedDims + d] = (uint8_t)bin[d];
            } else {
#pragma unroll
                for (int k = 0; k < 3; ++k) acc[k] += w[k];
            }
        }
    }
    if constexpr (!TRAIN) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double v = acc[k];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red[k][warp] = v;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double v = 0.0;
            for (int w = 0; w < kFixedThreads / 32; ++w) v += red[threadIdx.x][w];
            partial[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 3 + threadIdx.x] = v;
        }
    }
}

// Per-CTA sums of |w_k| (fixed order)
__global__ void fixed_abs_sum_kernel(const double* __restrict__ w, uint64_t n, double* __restrict__ partial)
{
    __shared__ double red[3][kFixedThreads / 32];
    double acc[3] = {0.0, 0.0, 0.0};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < 3; ++k) acc[k] += ::fabs(w[i * 3 + k]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int q = 0; q < kFixedThreads / 32; ++q) v += red[threadIdx.x][q];
        partial[blockIdx.x * 3 + threadIdx.x] = v;
    }
}

// score_i = sum_k weight_k |w_ik| / max(mean_k, tiny) into the |.| histograms of the Vegas
// partial layout [blocks][2 + 5*bins] (the first two slots zero) and the integer counts.
__global__ void fixed_score_hist_kernel(const double* __restrict__ w, const uint8_t* __restrict__ bins_in,
                                        uint64_t n, const double* __restrict__ abs_partial, int abs_blocks,
                                        double i1_weight, int bins, double* __restrict__ partial,
                                        int32_t* __restrict__ counts)
{
    extern __shared__ double hsm[];
    constexpr int D = kFixedDims;
    const int warps = kFixedThreads / 32;
    double* whist = hsm;                                           // [warps][D*bins]
    int32_t* cnt = reinterpret_cast<int32_t*>(whist + warps * D * bins);  // [D*bins]
    __shared__ double mean[3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < warps * D * bins; k += blockDim.x) whist[k] = 0.0;
    for (int k = threadIdx.x; k < D * bins; k += blockDim.x) cnt[k] = 0;
    if (threadIdx.x < 3) {
        double v = 0.0;
        for (int b = 0; b < abs_blocks; ++b) v += abs_partial[b * 3 + threadIdx.x];
        v /= (double)n;
        mean[threadIdx.x] = v > 2.2250738585072014e-308 ? v : 2.2250738585072014e-308;
    }
    __syncthreads();
    double* myhist = whist + warp * D * bins;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        const bool active = i < n;
        const unsigned mask = __ballot_sync(0xffffffffu, active);
        if (!active) continue;
        const double score = i1_weight * ::fabs(w[i * 3 + 0]) / mean[0] + ::fabs(w[i * 3 + 1]) / mean[1] +
                             ::fabs(w[i * 3 + 2]) / mean[2];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const int key = d * bins + bins_in[i * D + d];
            const unsigned peers = __match_any_sync(mask, key);
            const int rank = __popc(peers & ((1u << lane) - 1u));
            const int last = __reduce_max_sync(mask, rank);
            for (int k = 0; k <= last; ++k) {
                if (rank == k) myhist[key] += score;
                __syncwarp(mask);
            }
            atomicAdd(&cnt[key], 1);
        }
    }
    __syncthreads();
    double* out = partial + (size_t)blockIdx.x * (2 + D * bins);
    if (threadIdx.x == 0) {
        out[0] = 0.0;
        out[1] = 0.0;
    }
    for (int k = threadIdx.x; k < D * bins; k += blockDim.x) {
        double h = 0.0;
        for (int q = 0; q < warps; ++q) h += whist[q * D * bins + k];
        out[2 + k] = h;
        if (cnt[k]) atomicAdd(&counts[k], cnt[k]);
    }
}

// estimates[j][k] = (sum over CTAs of partial[b][k]) / n, fixed order
// One CTA per replicate: its CTA sums in CTA order.
__global__ void fixed_estimate_kernel(const double* __restrict__ partial, int blocks, uint64_t n,
                                      double* __restrict__ estimate)
{
    if (threadIdx.x >= 3) return;
    const double* p = partial + (size_t)blockIdx.x * blocks * 3;
    double v = 0.0;
    for (int b = 0; b < blocks; ++b) v += p[b * 3 + threadIdx.x];
    estimate[3 * blockIdx.x + threadIdx.x] = v / (double)n;
}

__global__ void fixed_grid_init_kernel(double* state, int D, int bins)
{
    for (int k = threadIdx.x; k < D * (bins + 1); k += blockDim.x) {
        const int b = k % (bins + 1);
        state[k] = b == bins ? 1.0 : (double)b / bins;
    }
    for (int k = threadIdx.x; k < kStSlots; k += blockDim.x) state[D * (bins + 1) + k] = 0.0;
}

__global__ void fixed_zero_counts_kernel(int32_t* counts, int n)
{
    for (int k = threadIdx.x; k < n; k += blockDim.x) counts[k] = 0;
}

}  // namespace dis

namespace {

int ffail(int code, const std::string& m) { return set_last_error(code, m.c_str()); }

int fcuda(cudaError_t e, const char* where)
{
    return ffail(NLO_ERR_CUDA, std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

struct FixedCarve {
    size_t dirs, w, b, partial, abs_partial, reduced, counts, total;
};

constexpr size_t kAl = 256;
size_t al(size_t v) { return (v + kAl - 1) & ~(kAl - 1); }

// CTAs of a launch over n samples: two lanes a sample (fixed_triple_kernel), up to four
// waves of three CTAs per SM.  The workspace carve and the launches both size by it.
int fixed_blocks(uint64_t n)
{
    static int sms = [] {
        int device = 0, v = 148;
        if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
        return v > 0 ? v : 148;
    }();
    const uint64_t by_n = (2 * n + dis::kFixedThreads - 1) / dis::kFixedThreads;
    const uint64_t cap = (uint64_t)4 * 3 * sms;
    const uint64_t b = by_n < cap ? by_n : cap;
    return (int)(b < 1 ? 1 : b);
}

FixedCarve fixed_carve(const nlo_fixed_sobol_options& o)
{
    const int rounds = o.training_rounds + o.replicates;
    const uint64_t most = (uint64_t)(o.training_samples > o.samples_per_replicate ? o.training_samples
                                                                                 : o.samples_per_replicate);
    const int blocks = fixed_blocks(most);
    FixedCarve c;
    c.dirs = 0;
    c.w = al(c.dirs + sizeof(SobolDirsArg) * (size_t)rounds);
    c.b = al(c.w + sizeof(double) * 3 * (size_t)o.training_samples);
    c.partial = al(c.b + (size_t)dis::kFixedDims * o.training_samples);
    // per-CTA partials: the training histograms, or all replicates' sums at once
    const size_t train_partial = (size_t)blocks * (2 + dis::kFixedDims * (size_t)o.bins);
    const size_t replicate_partial = (size_t)o.replicates * fixed_blocks((uint64_t)o.samples_per_replicate) * 3;
    c.abs_partial = al(c.partial + sizeof(double) * (train_partial > replicate_partial ? train_partial
                                                                                       : replicate_partial));
    c.reduced = al(c.abs_partial + sizeof(double) * 3 * (size_t)blocks);
    c.counts = al(c.reduced + sizeof(double) * (2 + dis::kFixedDims * (size_t)o.bins));
    c.total = al(c.counts + sizeof(int32_t) * dis::kFixedDims * (size_t)o.bins);
    return c;
}

template <typename T>
int run_fixed(const dis::DisArgs<T>& args, const dis::InnerRule& rule, const nlo_fixed_sobol_options& o,
              unsigned char* ws, const FixedCarve& c, double* grid_state, double* estimates, cudaStream_t s)
{
    using namespace dis;
    const FixedGeom g{args.maxr, o.bins, o.fold_angle ? 1 : 0};
    const SobolDirsArg* dirs = reinterpret_cast<const SobolDirsArg*>(ws + c.dirs);
    double* w = reinterpret_cast<double*>(ws + c.w);
    uint8_t* bb = reinterpret_cast<uint8_t*>(ws + c.b);
    double* partial = reinterpret_cast<double*>(ws + c.partial);
    double* abs_partial = reinterpret_cast<double*>(ws + c.abs_partial);
    double* reduced = reinterpret_cast<double*>(ws + c.reduced);
    int32_t* counts = reinterpret_cast<int32_t*>(ws + c.counts);
    const int stride = kFixedDims * (o.bins + 1) + kStSlots;
    fixed_grid_init_kernel<<<1, 256, 0, s>>>(grid_state, kFixedDims, o.bins);
    fixed_zero_counts_kernel<<<1, 256, 0, s>>>(counts, kFixedDims * o.bins);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fcuda(e, "fixed-Sobol init");
    const size_t hsmem =
        sizeof(double) * (kFixedThreads / 32) * kFixedDims * o.bins + sizeof(int32_t) * kFixedDims * o.bins;
    e = raise_dynamic_smem((const void*)fixed_score_hist_kernel, hsmem);
    if (e != cudaSuccess) return fcuda(e, "fixed-Sobol histogram attribute");
    const uint64_t nt = (uint64_t)o.training_samples;
    const int tb = fixed_blocks(nt);
    for (int r = 0; r < o.training_rounds; ++r) {
        fixed_triple_kernel<T, true><<<tb, kFixedThreads, 0, s>>>(args, rule, dirs, r, nt, grid_state, g, w, bb,
                                                                  nullptr);
        fixed_abs_sum_kernel<<<tb, kFixedThreads, 0, s>>>(w, nt, abs_partial);
        fixed_score_hist_kernel<<<tb, kFixedThreads, hsmem, s>>>(w, bb, nt, abs_partial, tb, o.i1_weight, o.bins,
                                                                  partial, counts);
        e = cudaGetLastError();
        if (e != cudaSuccess) return fcuda(e, "fixed-Sobol training launch");
        e = dis_launch_reduce_finalize(kFixedDims, o.bins, 1, tb, partial, reduced, counts, grid_state, stride, nt, 1,
                                       1, 0.0, 0.0, s);
        if (e != cudaSuccess) return fcuda(e, "fixed-Sobol grid adaptation");
    }
    const uint64_t nr = (uint64_t)o.samples_per_replicate;
    const int rb = fixed_blocks(nr);
    // the replicates are independent (own Sobol seeds, the frozen grid): one launch
    fixed_triple_kernel<T, false><<<dim3(rb, o.replicates), kFixedThreads, 0, s>>>(
        args, rule, dirs, o.training_rounds, nr, grid_state, g, nullptr, nullptr, partial);
    fixed_estimate_kernel<<<o.replicates, 32, 0, s>>>(partial, rb, nr, estimates);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fcuda(e, "fixed-Sobol replicate launch");
    return NLO_OK;
}

}  // namespace

bool dis_fixed_check(const nlo_fixed_sobol_options* o, std::string& why)
{
    if (!o) { why = "options is NULL"; return false; }
    auto pow2 = [](int64_t v) { return v >= 2 && (v & (v - 1)) == 0; };
    if (!pow2(o->training_samples) || !pow2(o->samples_per_replicate)) {
        why = "Sobol sample counts must be powers of two greater than one";
        return false;
    }
    if (o->training_rounds < 1 || o->replicates < 2) {
        why = "training rounds must be positive; replicates must exceed one";
        return false;
    }
    if (o->training_rounds + o->replicates > 64) { why = "at most 64 training rounds and replicates"; return false; }
    if (o->bins < 2 || o->bins > 256) { why = "bins must lie in 2..256"; return false; }
    if (o->training_samples > (int64_t(1) << 30) || o->samples_per_replicate > (int64_t(1) << 30)) {
        why = "Sobol index range exceeds 2^30";
        return false;
    }
    if (o->inner_points < 8 || o->inner_points > dis::kMaxInner) { why = "the inner rule needs 8..128 points"; return false; }
    if (o->precision != NLO_PRECISION_MIXED && o->precision != NLO_PRECISION_FP64) { why = "unknown precision"; return false; }
    return true;
}

size_t dis_fixed_workspace_bytes(const nlo_fixed_sobol_options& o) { return fixed_carve(o).total; }

int dis_run_fixed(int precision, const void* args, const dis::InnerRule& rule, const nlo_fixed_sobol_options& o,
                  void* workspace, double* grid_state, double* estimates, cudaStream_t s)
{
    const FixedCarve c = fixed_carve(o);
    unsigned char* ws = static_cast<unsigned char*>(workspace);
    if (precision == NLO_PRECISION_FP64)
        return run_fixed(*static_cast<const dis::DisArgs<double>*>(args), rule, o, ws, c, grid_state, estimates, s);
    return run_fixed(*static_cast<const dis::DisArgs<float>*>(args), rule, o, ws, c, grid_state, estimates, s);
}

}  // namespace nlo
