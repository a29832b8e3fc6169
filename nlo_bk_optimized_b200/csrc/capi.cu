// extern "C" entry points of libnlo_b200.so (declared in include/nlo_b200.h):
// argument checks, workspace carving and the host-side stage sequence.  Nothing
// here allocates device memory and nothing synchronises the stream.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace nlo {

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& message)
{
    g_last_error = message;
    return code;
}

int cuda_fail(cudaError_t e, const char* where)
{
    return fail(NLO_ERR_CUDA, std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

// Gauss-Legendre nodes on [-1, 1] in ascending order by Newton iteration on P_n
// (the same construction as numerics/integration.py:781-801).
void gauss_legendre(int n, double* x, double* w)
{
    for (int i = 0; i < n; ++i) {
        double t = std::cos(kPi * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = t;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (t * p1 - p0) / (t * t - 1.0);
            const double dt = p1 / dp;
            t -= dt;
            if (std::fabs(dt) < 1e-16) break;
        }
        double p0 = 1.0, p1 = t;
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        dp = n * (t * p1 - p0) / (t * t - 1.0);
        x[n - 1 - i] = t;
        w[n - 1 - i] = 2.0 / ((1.0 - t * t) * dp * dp);
    }
}

size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

// Workspace layout of one right-hand-side evaluation.
size_t rhs_bytes(int points, size_t* offsets /*[10] or NULL*/)
{
    size_t o = 0;
    size_t off[10];
    off[0] = o; o = align_up(o + sizeof(double) * spline_doubles(points));
    off[1] = o; o = align_up(o + sizeof(int32_t) * (size_t)points);
    off[2] = o; o = align_up(o + sizeof(int32_t) * 4);
    off[3] = o; o = align_up(o + sizeof(double) * (size_t)points);
    off[4] = o; o = align_up(o + sizeof(double) * 3 * (size_t)points);
    off[5] = o; o = align_up(o + sizeof(double) * 3 * (size_t)points * (size_t)k2kf_max_blocks());
    off[6] = o; o = align_up(o + sizeof(double) * 2 * (size_t)points);
    off[7] = o; o = align_up(o + sizeof(double) * kc_weights_doubles(points));
    off[8] = o; o = align_up(o + sizeof(int32_t) * (size_t)points);
    off[9] = o; o = align_up(o + sizeof(int32_t) * 4);
    if (offsets) std::memcpy(offsets, off, sizeof(off));
    return o;
}

RhsBuffers carve(void* ws, int points)
{
    size_t off[10];
    rhs_bytes(points, off);
    char* base = static_cast<char*>(ws);
    RhsBuffers b;
    b.spline = reinterpret_cast<double*>(base + off[0]);
    b.active = reinterpret_cast<int32_t*>(base + off[1]);
    b.count = reinterpret_cast<int32_t*>(base + off[2]);
    b.k1 = reinterpret_cast<double*>(base + off[3]);
    b.k2kf = reinterpret_cast<double*>(base + off[4]);
    b.partial = reinterpret_cast<double*>(base + off[5]);
    b.factor = reinterpret_cast<double*>(base + off[6]);
    b.kc = reinterpret_cast<double*>(base + off[7]);
    b.k1_active = reinterpret_cast<int32_t*>(base + off[8]);
    b.k1_count = reinterpret_cast<int32_t*>(base + off[9]);
    b.k2kf_blocks = k2kf_max_blocks();
    return b;
}

// A side stream for K1: K1 and K2+Kf read the same spline and active list and write
// different buffers, so K1 runs beside K2+Kf and its last, partly filled wave of CTAs
// overlaps the start of K2+Kf instead of idling most SMs.  One per evolve/rhs call.
struct SideStream {
    cudaStream_t aux = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    bool ok = false;
    SideStream()
    {
        ok = cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&join, cudaEventDisableTiming) == cudaSuccess;
        if (!ok) cudaGetLastError();  // fall back to one stream
    }
    ~SideStream()
    {
        if (join) cudaEventDestroy(join);
        if (fork) cudaEventDestroy(fork);
        if (aux) cudaStreamDestroy(aux);
    }
    SideStream(const SideStream&) = delete;
    SideStream& operator=(const SideStream&) = delete;
};

// One rapidity step recorded as a CUDA graph and replayed for every later step: the step's
// launches (4 x (spline refit, active list, K1 on the side stream, K2+Kf, its finalize,
// assembly) + the stage combinations for RK4) then cost one graph launch, and the device runs
// them without the per-launch gaps.  The recorded step reads and writes one fixed row (the
// last stage combination runs in place, element by element), so the same graph serves every
// step; the caller copies the row out to the table after each replay.  Capture runs on a
// private stream in thread-local mode, so that the caller's stream (which may be the legacy
// default stream) and other threads are untouched; if recording fails for any reason the
// caller launches the step's kernels one by one instead.
struct StepGraph {
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    StepGraph() = default;
    StepGraph(const StepGraph&) = delete;
    StepGraph& operator=(const StepGraph&) = delete;
    ~StepGraph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (cap) cudaStreamDestroy(cap);
    }
    // record(stream) enqueues the step on `stream`; true when a replayable graph came out
    template <class F>
    bool capture(F record)
    {
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
            cap = nullptr;
            cudaGetLastError();
            return false;
        }
        if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        const int rc = record(cap);
        const cudaError_t end = cudaStreamEndCapture(cap, &graph);
        if (rc != NLO_OK || end != cudaSuccess || !graph ||
            cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            cudaGetLastError();
            if (exec) cudaGraphExecDestroy(exec);
            exec = nullptr;
            return false;
        }
        return true;
    }
};

// Measured on the B200 (RK4, 2^14..2^20 samples per parent): with 200 and 400 points a
// replayed step took 0.74-0.98 of the launched one (0.95 at the 400-point, 2^20-sample
// evolution); with 100 to 160 points, where the K2+Kf launch has CTAs of 128 or 160 lanes,
// five to seven per SM, up to 1.6 times as long.  So grids of up to 192 points (the largest
// with 192-lane CTAs, not measured) launch every step.
inline bool replay_pays(int points) { return points > 192; }

int run_rhs(const nlo_bk_params& p, const double* r, const double* N, int points, const SobolDirsArg& dirs,
            uint64_t samples, const nlo_bk_box& box, double* dndy, double* k1_out, double* k2kf_out,
            const RhsBuffers& b, bool factor_ready, cudaStream_t stream, int shard = 0, int shards = 1,
            const double* hist_y = nullptr, const double* hist_N = nullptr, int rows = 0,
            const SideStream* side = nullptr, const BkVegasCall* vegas = nullptr)
{
    cudaError_t e;
    K1History history;
    if (p.kinematical_constraint) {
        if ((e = launch_kc_weights(r, points, b.kc, stream)) != cudaSuccess) return cuda_fail(e, "kc weights");
        history.N = hist_N;
        history.y = hist_y;
        history.weights = b.kc;
        history.rows = rows;
        history.on = true;
    }
    if ((e = launch_splines(r, single_row(N), points, 1, p.force_positive, b.factor, factor_ready ? 0 : 1, b.spline,
                            stream)) !=
        cudaSuccess)
        return cuda_fail(e, "splines");
    // Sobol QMC: K2+Kf takes every active parent (a shard owns a range of Sobol indices), K1
    // the active parents i with i % shards == shard.  Vegas: both take the shard's parents.
    const bool split_samples = vegas == nullptr;
    if ((e = launch_active(single_row(N), points, 1, split_samples ? 0 : shard, split_samples ? 1 : shards, b.active,
                           b.count,
                           stream)) != cudaSuccess)
        return cuda_fail(e, "active");
    const int32_t* k1_active = b.active;
    const int32_t* k1_count = b.count;
    if (shards > 1 && split_samples) {
        if ((e = launch_active(single_row(N), points, 1, shard, shards, b.k1_active, b.k1_count, stream)) !=
            cudaSuccess)
            return cuda_fail(e, "active");
        k1_active = b.k1_active;
        k1_count = b.k1_count;
    }
    const bool beside = side && side->ok;
    cudaStream_t k1_stream = stream;
    if (beside) {
        if ((e = cudaEventRecord(side->fork, stream)) != cudaSuccess) return cuda_fail(e, "fork");
        if ((e = cudaStreamWaitEvent(side->aux, side->fork, 0)) != cudaSuccess) return cuda_fail(e, "fork");
        k1_stream = side->aux;
    }
    if ((e = launch_k1(p, r, points, b.spline, k1_active, k1_count, b.k1, k1_stream, history)) != cudaSuccess)
        return cuda_fail(e, "k1");
    if (beside && (e = cudaEventRecord(side->join, side->aux)) != cudaSuccess) return cuda_fail(e, "join");
    // orders without NLO kernels (Order.has_nlo_kernels, bk/config.py:44-50) take no K2 + Kf:
    // zero samples clear the sums and launch nothing
    double k2kf_factor = 0.0;
    if (vegas) {
        if (order_has_nlo(p.order)) {
            if ((e = launch_k2kf_vegas(p, r, N, points, b.spline, shard, shards, dirs, box, *vegas, b.k2kf, stream)) !=
                cudaSuccess)
                return cuda_fail(e, "k2kf vegas");
            k2kf_factor = 1.0;  // the Vegas values are integrals already
        } else if ((e = cudaMemsetAsync(b.k2kf, 0, sizeof(double) * 3 * (size_t)points, stream)) != cudaSuccess) {
            return cuda_fail(e, "k2kf clear");
        }
    } else {
        const uint64_t nlo_samples = order_has_nlo(p.order) ? samples : 0;
        // this shard's Sobol indices [first, last) of the nlo_samples points; the sums are
        // divided by nlo_samples, so the shards' right-hand sides add up to the whole one
        const uint64_t first = nlo_samples * (uint64_t)shard / (uint64_t)shards;
        const uint64_t last = nlo_samples * (uint64_t)(shard + 1) / (uint64_t)shards;
        if ((e = launch_k2kf(p, r, points, b.spline, b.active, b.count, dirs, first, last - first, box, b.k2kf,
                             b.partial, b.k2kf_blocks, stream)) != cudaSuccess)
            return cuda_fail(e, "k2kf");
        k2kf_factor = nlo_samples ? 1.0 / (double)nlo_samples : 0.0;
    }
    if (beside && (e = cudaStreamWaitEvent(stream, side->join, 0)) != cudaSuccess) return cuda_fail(e, "join");
    // the replica refinement reads this right-hand side's K1
    if (vegas && order_has_nlo(p.order) && vegas->options.replicas > 0 &&
        (e = launch_k2kf_vegas_refine(p, r, N, points, b.spline, box, *vegas, b.k1, b.k2kf, stream)) != cudaSuccess)
        return cuda_fail(e, "k2kf vegas replicas");
    if ((e = launch_assemble(b.k1, b.k2kf, points, k2kf_factor, dndy, k2kf_out, stream)) != cudaSuccess)
        return cuda_fail(e, "assemble");
    if (k1_out) {
        if ((e = cudaMemcpyAsync(k1_out, b.k1, sizeof(double) * points, cudaMemcpyDeviceToDevice, stream)) !=
            cudaSuccess)
            return cuda_fail(e, "k1 copy");
    }
    return NLO_OK;
}

// The stage sequence of one rapidity step (_bk_steps with its Euler, Kutta RK3 and RK4 steppers,
// bk/evolution.py:85-236): rhs(src, k) evaluates the right-hand side of the stage input src
// (-1: the step's row, 0: the stage row) into derivative k; comb(nk, ks, coef, dst) forms
// row + sum_j coef[j] k[ks[j]] into the stage row (dst 0) or the next row (dst 1).
template <class Rhs, class Comb>
int step_sequence(int stepper, double step, Rhs rhs, Comb comb)
{
    int rc;
    if (stepper == NLO_STEPPER_EULER) {
        if ((rc = rhs(-1, 0)) != NLO_OK) return rc;
        const int k0[1] = {0};
        const double c[1] = {step};
        return comb(1, k0, c, 1);
    }
    if (stepper == NLO_STEPPER_RK3) {
        // Kutta RK3 (bk/evolution.py:204-236)
        if ((rc = rhs(-1, 0)) != NLO_OK) return rc;
        const int k0[1] = {0}, k01[2] = {0, 1}, k012[3] = {0, 1, 2};
        const double c1[1] = {0.5 * step};
        if ((rc = comb(1, k0, c1, 0)) != NLO_OK) return rc;
        if ((rc = rhs(0, 1)) != NLO_OK) return rc;
        const double c2[2] = {-step, 2.0 * step};
        if ((rc = comb(2, k01, c2, 0)) != NLO_OK) return rc;
        if ((rc = rhs(0, 2)) != NLO_OK) return rc;
        const double c3[3] = {step / 6.0, 4.0 * step / 6.0, step / 6.0};
        return comb(3, k012, c3, 1);
    }
    // classical RK4
    if ((rc = rhs(-1, 0)) != NLO_OK) return rc;
    const int k0[1] = {0}, k1[1] = {1}, k2[1] = {2}, k0123[4] = {0, 1, 2, 3};
    const double c1[1] = {0.5 * step};
    if ((rc = comb(1, k0, c1, 0)) != NLO_OK) return rc;
    if ((rc = rhs(0, 1)) != NLO_OK) return rc;
    if ((rc = comb(1, k1, c1, 0)) != NLO_OK) return rc;
    if ((rc = rhs(0, 2)) != NLO_OK) return rc;
    const double c3[1] = {step};
    if ((rc = comb(1, k2, c3, 0)) != NLO_OK) return rc;
    if ((rc = rhs(0, 3)) != NLO_OK) return rc;
    const double c4[4] = {step / 6.0, 2.0 * step / 6.0, 2.0 * step / 6.0, step / 6.0};
    return comb(4, k0123, c4, 1);
}

}  // namespace

bool check_params(const nlo_bk_params* p, std::string& why)
{
    if (!p) { why = "params is NULL"; return false; }
    if (!(p->nc > 0)) { why = "NC must be positive"; return false; }
    if (!(p->nf == 0.0 || p->nf == 3.0 || p->nf == 5.0)) { why = "NF must be 0, 3 or 5"; return false; }
    if (p->order < NLO_ORDER_NLO_RESUM_DLOG_SLOG || p->order > NLO_ORDER_LO) { why = "unknown order"; return false; }
    if (p->rc_lo < NLO_RC_LO_BALITSKY || p->rc_lo > NLO_RC_LO_BEUF) { why = "unknown RC_LO"; return false; }
    if (p->resum_rc < NLO_RESUM_RC_SMALLEST || p->resum_rc > NLO_RESUM_RC_FIXED) { why = "unknown RESUM_RC"; return false; }
    if (p->rc_nlo != NLO_RC_NLO_SMALLEST && p->rc_nlo != NLO_RC_NLO_PARENT) { why = "unknown RC_NLO"; return false; }
    if (!(p->lambda_qcd > 0) || !(p->c2 > 0) || !(p->ksub > 0)) { why = "LambdaQCD, C2 and KSUB must be positive"; return false; }
    if (p->precision != NLO_PRECISION_MIXED && p->precision != NLO_PRECISION_FP64) { why = "unknown precision"; return false; }
    return true;
}

bool check_dirs(const nlo_sobol_dirs* d, int need, std::string& why)
{
    if (!d) { why = "dirs is NULL"; return false; }
    if (d->dims < need || d->dims > 8) { why = "Sobol dimension count out of range"; return false; }
    for (int j = 0; j < d->dims; ++j) {
        if (d->shift[j] >= (1u << 30)) { why = "Sobol shift exceeds 30 bits"; return false; }
        for (int k = 0; k < 30; ++k)
            if (d->state[j][k] >= (1u << 30)) { why = "Sobol direction number exceeds 30 bits"; return false; }
    }
    return true;
}

SobolDirsArg to_arg(const nlo_sobol_dirs* d)
{
    SobolDirsArg a;
    std::memset(&a, 0, sizeof(a));
    a.dims = d->dims;
    std::memcpy(a.state, d->state, sizeof(a.state));
    std::memcpy(a.shift, d->shift, sizeof(a.shift));
    return a;
}

const K1Rule& k1_rule()
{
    static K1Rule rule = [] {
        K1Rule q;
        gauss_legendre(8, q.x8, q.w8);
        gauss_legendre(24, q.x24, q.w24);
        return q;
    }();
    return rule;
}

int set_last_error(int code, const char* message) { return fail(code, message); }

void gauss_legendre_rule(int n, double* x, double* w) { gauss_legendre(n, x, w); }

cudaError_t raise_dynamic_smem(const void* func, size_t bytes)
{
    // The limit is a property of the kernel on the device, shared by every host thread:
    // only ever raise it, so that a launch prepared by one thread is never invalidated by
    // another thread lowering the limit for a smaller launch of the same kernel.
    static std::mutex lock;
    static std::map<std::pair<int, const void*>, size_t> limits;
    if (bytes <= 48 * 1024) return cudaSuccess;  // within the default limit
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> guard(lock);
    size_t& current = limits[{device, func}];
    if (bytes <= current) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) current = bytes;
    return e;
}

// buffer size a caller provides to nlo_bk_splines: coefficients plus factorisation scratch
cudaError_t prefer_shared_carveout(const void* func)
{
    static std::mutex lock;
    static std::set<std::pair<int, const void*>> done;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> guard(lock);
    if (done.count({device, func})) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e == cudaSuccess) done.insert({device, func});
    return e;
}

size_t spline_buffer_doubles(int points) { return spline_doubles(points) + 2 * (size_t)points; }

int k2kf_max_blocks()
{
    static int blocks = [] {
        int device = 0, sms = 148;
        if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        return 4 * (sms > 0 ? sms : 148);
    }();
    return blocks;
}

}  // namespace nlo

using namespace nlo;

extern "C" {

const char* nlo_last_error(void) { return g_last_error.c_str(); }

int nlo_abi_version(void) { return 1; }

int nlo_sobol_draw(const nlo_sobol_dirs* dirs, int64_t offset, int64_t n, int32_t precision, void* out, void* stream)
{
    std::string why;
    if (!check_dirs(dirs, 1, why)) return fail(NLO_ERR_INVALID, why);
    if (offset < 0 || n < 0 || offset + n > (int64_t(1) << 30)) return fail(NLO_ERR_INVALID, "Sobol index range exceeds 2^30");
    if (precision != NLO_PRECISION_MIXED && precision != NLO_PRECISION_FP64) return fail(NLO_ERR_INVALID, "unknown precision");
    if (n == 0) return NLO_OK;
    if (!out) return fail(NLO_ERR_INVALID, "out is NULL");
    cudaError_t e = launch_sobol(to_arg(dirs), (uint64_t)offset, (uint64_t)n, precision, out, (cudaStream_t)stream);
    return e == cudaSuccess ? NLO_OK : cuda_fail(e, "sobol");
}

size_t nlo_bk_spline_doubles(int32_t points) { return points >= 2 ? spline_buffer_doubles(points) : 0; }

int nlo_bk_splines(const double* r, const double* N, int32_t points, int32_t force_positive, double* spline, void* stream)
{
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "a cubic spline requires 3..4096 points");
    if (!r || !N || !spline) return fail(NLO_ERR_INVALID, "NULL buffer");
    // the factorisation scratch is the tail of the caller's spline buffer (nlo_bk_spline_doubles)
    double* factor = spline + spline_doubles(points);
    cudaError_t e = launch_splines(r, single_row(N), points, 1, force_positive, factor, 1, spline, (cudaStream_t)stream);
    return e == cudaSuccess ? NLO_OK : cuda_fail(e, "splines");
}

int nlo_bk_active(const double* N, int32_t points, int32_t* active, int32_t* count, void* stream)
{
    if (points < 1) return fail(NLO_ERR_INVALID, "points must be positive");
    if (!N || !active || !count) return fail(NLO_ERR_INVALID, "NULL buffer");
    cudaError_t e = launch_active(single_row(N), points, 1, 0, 1, active, count, (cudaStream_t)stream);
    return e == cudaSuccess ? NLO_OK : cuda_fail(e, "active");
}

int nlo_bk_k1(const nlo_bk_params* params, const double* r, int32_t points, const double* spline,
              const int32_t* active, const int32_t* count, double* out, void* stream)
{
    std::string why;
    if (!check_params(params, why)) return fail(NLO_ERR_INVALID, why);
    if (params->kinematical_constraint)
        return fail(NLO_ERR_INVALID, "the kinematical constraint reads the amplitude history: use nlo_bk_rhs_history "
                                     "or nlo_bk_evolve_history");
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "points must be 3..4096");
    if (!r || !spline || !active || !count || !out) return fail(NLO_ERR_INVALID, "NULL buffer");
    cudaError_t e = launch_k1(*params, r, points, spline, active, count, out, (cudaStream_t)stream);
    return e == cudaSuccess ? NLO_OK : cuda_fail(e, "k1");
}

size_t nlo_bk_k2kf_workspace_bytes(int32_t points)
{
    if (points < 1) return 0;
    return sizeof(double) * 3 * (size_t)points * (size_t)k2kf_max_blocks();
}

int nlo_bk_k2kf(const nlo_bk_params* params, const double* r, int32_t points, const double* spline,
                const int32_t* active, const int32_t* count, const nlo_sobol_dirs* dirs, int64_t offset,
                int64_t samples, const nlo_bk_box* box, double* out, void* workspace, size_t workspace_bytes,
                void* stream)
{
    std::string why;
    if (!check_params(params, why)) return fail(NLO_ERR_INVALID, why);
    if (!check_dirs(dirs, 4, why)) return fail(NLO_ERR_INVALID, why);
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "points must be 3..4096");
    if (!r || !spline || !active || !count || !out || !box) return fail(NLO_ERR_INVALID, "NULL buffer");
    if (offset < 0 || samples < 0 || offset + samples > (int64_t(1) << 30))
        return fail(NLO_ERR_INVALID, "Sobol index range exceeds 2^30");
    if (!workspace || workspace_bytes < nlo_bk_k2kf_workspace_bytes(points))
        return fail(NLO_ERR_WORKSPACE, "workspace too small for nlo_bk_k2kf");
    cudaError_t e = launch_k2kf(*params, r, points, spline, active, count, to_arg(dirs), (uint64_t)offset,
                                (uint64_t)samples, *box, out, static_cast<double*>(workspace), k2kf_max_blocks(),
                                (cudaStream_t)stream);
    return e == cudaSuccess ? NLO_OK : cuda_fail(e, "k2kf");
}

size_t nlo_bk_rhs_workspace_bytes(int32_t points)
{
    if (points < 3) return 0;
    // one right-hand side plus five stage rows for the steppers and the row a recorded step
    // advances
    return rhs_bytes(points, nullptr) + align_up(sizeof(double) * 6 * (size_t)points);
}

int nlo_bk_rhs(const nlo_bk_params* params, const double* r, const double* N, int32_t points,
               const nlo_sobol_dirs* dirs, int64_t samples, const nlo_bk_box* box, double* dndy, double* k1,
               double* k2kf, void* workspace, size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!check_params(params, why)) return fail(NLO_ERR_INVALID, why);
    if (params->kinematical_constraint)
        return fail(NLO_ERR_INVALID, "the kinematical constraint reads the amplitude history: use nlo_bk_rhs_history "
                                     "or nlo_bk_evolve_history");
    if (!check_dirs(dirs, 4, why)) return fail(NLO_ERR_INVALID, why);
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "points must be 3..4096");
    if (!r || !N || !dndy || !box) return fail(NLO_ERR_INVALID, "NULL buffer");
    if (samples < 0 || samples > (int64_t(1) << 30)) return fail(NLO_ERR_INVALID, "samples out of range");
    if (!workspace || workspace_bytes < nlo_bk_rhs_workspace_bytes(points))
        return fail(NLO_ERR_WORKSPACE, "workspace too small for nlo_bk_rhs");
    const RhsBuffers b = carve(workspace, points);
    const SideStream side;
    return run_rhs(*params, r, N, points, to_arg(dirs), (uint64_t)samples, *box, dndy, k1, k2kf, b, false,
                   (cudaStream_t)stream, 0, 1, nullptr, nullptr, 0, &side);
}

int nlo_bk_rhs_shard(const nlo_bk_params* params, const double* r, const double* N, int32_t points, int32_t shard,
                     int32_t shards, const nlo_sobol_dirs* dirs, int64_t samples, const nlo_bk_box* box, double* dndy,
                     void* workspace, size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!check_params(params, why)) return fail(NLO_ERR_INVALID, why);
    if (params->kinematical_constraint)
        return fail(NLO_ERR_INVALID, "the kinematical constraint reads the amplitude history: use nlo_bk_rhs_history "
                                     "or nlo_bk_evolve_history");
    if (!check_dirs(dirs, 4, why)) return fail(NLO_ERR_INVALID, why);
    if (shards < 1 || shard < 0 || shard >= shards) return fail(NLO_ERR_INVALID, "shard must lie in [0, shards)");
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "points must be 3..4096");
    if (!r || !N || !dndy || !box) return fail(NLO_ERR_INVALID, "NULL buffer");
    if (samples < 0 || samples > (int64_t(1) << 30)) return fail(NLO_ERR_INVALID, "samples out of range");
    if (!workspace || workspace_bytes < nlo_bk_rhs_workspace_bytes(points))
        return fail(NLO_ERR_WORKSPACE, "workspace too small for nlo_bk_rhs_shard");
    const RhsBuffers b = carve(workspace, points);
    const SideStream side;
    return run_rhs(*params, r, N, points, to_arg(dirs), (uint64_t)samples, *box, dndy, nullptr, nullptr, b, false,
                   (cudaStream_t)stream, shard, shards, nullptr, nullptr, 0, &side);
}

int nlo_bk_stage(const double* N, const double* const* k, const double* coef, int32_t nk, int32_t points,
                 int32_t clamp, double* out, uint32_t* status, void* stream)
{
    if (!N || !k || !coef || !out) return fail(NLO_ERR_INVALID, "NULL buffer");
    if (nk < 1 || nk > 4) return fail(NLO_ERR_INVALID, "nk must be 1..4");
    if (points < 1) return fail(NLO_ERR_INVALID, "points must be positive");
    for (int j = 0; j < nk; ++j)
        if (!k[j]) return fail(NLO_ERR_INVALID, "NULL stage derivative");
    cudaError_t e = launch_axpy_stage(N, k, coef, nk, points, out, clamp ? 1 : 0, status, (cudaStream_t)stream);
    return e == cudaSuccess ? NLO_OK : cuda_fail(e, "stage");
}

int nlo_bk_rhs_history(const nlo_bk_params* params, const double* r, int32_t points, const double* hist_y,
                       const double* hist_N, int32_t rows, const nlo_sobol_dirs* dirs, int64_t samples,
                       const nlo_bk_box* box, double* dndy, double* k1, double* k2kf, void* workspace,
                       size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!check_params(params, why)) return fail(NLO_ERR_INVALID, why);
    if (!check_dirs(dirs, 4, why)) return fail(NLO_ERR_INVALID, why);
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "points must be 3..4096");
    if (rows < 1) return fail(NLO_ERR_INVALID, "the history needs at least one row");
    if (!r || !hist_y || !hist_N || !dndy || !box) return fail(NLO_ERR_INVALID, "NULL buffer");
    if (samples < 0 || samples > (int64_t(1) << 30)) return fail(NLO_ERR_INVALID, "samples out of range");
    if (!workspace || workspace_bytes < nlo_bk_rhs_workspace_bytes(points))
        return fail(NLO_ERR_WORKSPACE, "workspace too small for nlo_bk_rhs_history");
    const RhsBuffers b = carve(workspace, points);
    const double* N = hist_N + (size_t)(rows - 1) * points;
    const SideStream side;
    return run_rhs(*params, r, N, points, to_arg(dirs), (uint64_t)samples, *box, dndy, k1, k2kf, b, false,
                   (cudaStream_t)stream, 0, 1, hist_y, hist_N, rows, &side);
}

// Rows first+1..first+steps of `table` from row `first` (the loop of _bk_steps,
// bk/evolution.py:85-159).  y (device, may be NULL without the kinematical constraint):
// the rapidities of all rows, read as the constraint's history.
static int evolve_rows(const nlo_bk_params* params, const double* r, int32_t points, const double* y, int32_t first,
                int32_t steps, double step, int32_t stepper, const nlo_sobol_dirs* dirs, int64_t samples,
                const nlo_bk_box* box, double* table, uint32_t* status, void* workspace, size_t workspace_bytes,
                void* stream, const BkVegasCall* vegas = nullptr)
{
    std::string why;
    if (!check_params(params, why)) return fail(NLO_ERR_INVALID, why);
    if (!check_dirs(dirs, 4, why)) return fail(NLO_ERR_INVALID, why);
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "points must be 3..4096");
    if (steps < 0 || first < 0) return fail(NLO_ERR_INVALID, "steps and first must be non-negative");
    if (!(step > 0) || !std::isfinite(step)) return fail(NLO_ERR_INVALID, "step must be positive");
    if (stepper != NLO_STEPPER_EULER && stepper != NLO_STEPPER_RK3 && stepper != NLO_STEPPER_RK4)
        return fail(NLO_ERR_INVALID, "unknown stepper");
    if (params->kinematical_constraint && stepper != NLO_STEPPER_EULER)
        return fail(NLO_ERR_INVALID, "the kinematical constraint requires the Euler stepper");
    if (params->kinematical_constraint && !y) return fail(NLO_ERR_INVALID, "the kinematical constraint needs y");
    if (!r || !table || !status || !box) return fail(NLO_ERR_INVALID, "NULL buffer");
    if (samples < 0 || samples > (int64_t(1) << 30)) return fail(NLO_ERR_INVALID, "samples out of range");
    if (!workspace || workspace_bytes < nlo_bk_rhs_workspace_bytes(points))
        return fail(NLO_ERR_WORKSPACE, "workspace too small for nlo_bk_evolve");
    cudaStream_t s = (cudaStream_t)stream;
    const RhsBuffers b = carve(workspace, points);
    double* stage = reinterpret_cast<double*>(static_cast<char*>(workspace) + rhs_bytes(points, nullptr));
    double* kk[4] = {stage, stage + points, stage + 2 * points, stage + 3 * points};
    double* tmp = stage + 4 * points;
    double* cur = stage + 5 * points;  // the row a recorded step advances in place
    const SobolDirsArg dirs_arg = to_arg(dirs);
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "status reset");
    const int clamp = params->force_positive ? 1 : 0;
    const SideStream side;
    // the spline factorisation depends on the grid only: form it on the first stage
    bool factor_ready = false;
    // the steps of a fixed-step Sobol evolution are all alike: after the first (launched one
    // by one, which also forms the factorisation and sets every kernel attribute) one step is
    // recorded and replayed; the kinematical constraint (its history grows) and Vegas (its
    // rounds depend on convergence checks) launch every step
    const bool replay = !params->kinematical_constraint && !vegas && steps > 1 && replay_pays(points);
    StepGraph graph;
    bool recorded = false;
    auto step_from = [&](const double* N, double* next, int it, cudaStream_t st) {
        auto rhs = [&](int src, int k) {
            const int code = run_rhs(*params, r, src < 0 ? N : tmp, points, dirs_arg, (uint64_t)samples, *box, kk[k],
                                     nullptr, nullptr, b, factor_ready, st, 0, 1, y, table, it + 1, &side, vegas);
            factor_ready = true;
            return code;
        };
        auto comb = [&](int nk, const int* ks, const double* coef, int dst) {
            const double* kp[4];
            for (int j = 0; j < nk; ++j) kp[j] = kk[ks[j]];
            const cudaError_t err = launch_axpy_stage(N, kp, coef, nk, points, dst ? next : tmp, dst ? clamp : 0,
                                                      dst ? status : nullptr, st);
            return err == cudaSuccess ? NLO_OK : cuda_fail(err, "stage");
        };
        return step_sequence(stepper, step, rhs, comb);
    };
    const size_t row_bytes = sizeof(double) * (size_t)points;
    for (int it = first; it < first + steps; ++it) {
        const double* N = table + (size_t)it * points;
        double* next = table + (size_t)(it + 1) * points;
        if (replay && it == first + 1) {
            recorded = graph.capture([&](cudaStream_t st) { return step_from(cur, cur, it, st); });
            if (recorded && (e = cudaMemcpyAsync(cur, N, row_bytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
                return cuda_fail(e, "step row");
        }
        if (recorded) {
            if ((e = cudaGraphLaunch(graph.exec, s)) != cudaSuccess) return cuda_fail(e, "step graph");
            if ((e = cudaMemcpyAsync(next, cur, row_bytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
                return cuda_fail(e, "step row");
            continue;
        }
        const int rc = step_from(N, next, it, s);
        if (rc != NLO_OK) return rc;
    }
    return NLO_OK;
}

// Workspace of a multi-set evolution: per set the spline tables, their factorisation, the
// active list and count, K1, the K2+Kf sums, five stage rows and the row a recorded step
// advances; the K2+Kf partial sums of the layout; the set table.
static size_t sets_bytes(int points, int sets, const SetsLayout& L, size_t* offsets /*[9] or NULL*/)
{
    const size_t S = (size_t)sets, n = (size_t)points;
    size_t o = 0, off[9];
    off[0] = o; o = align_up(o + sizeof(double) * S * spline_doubles(points));
    off[1] = o; o = align_up(o + sizeof(double) * S * 2 * n);
    off[2] = o; o = align_up(o + sizeof(int32_t) * S * n);
    off[3] = o; o = align_up(o + sizeof(int32_t) * S);
    off[4] = o; o = align_up(o + sizeof(double) * S * n);
    off[5] = o; o = align_up(o + sizeof(double) * S * 3 * n);
    off[6] = o; o = align_up(o + sizeof(double) * sets_partial_doubles(L));
    off[7] = o; o = align_up(o + sizeof(double) * 6 * S * n);
    off[8] = o; o = align_up(o + sizeof(SetTable));
    if (offsets) std::memcpy(offsets, off, sizeof(off));
    return o;
}

int nlo_bk_evolve(const nlo_bk_params* params, const double* r, int32_t points, int32_t steps, double step,
                  int32_t stepper, const nlo_sobol_dirs* dirs, int64_t samples, const nlo_bk_box* box,
                  double* table, uint32_t* status, void* workspace, size_t workspace_bytes, void* stream)
{
    if (params && params->kinematical_constraint)
        return fail(NLO_ERR_INVALID, "the kinematical constraint reads the amplitude history: use "
                                     "nlo_bk_evolve_history");
    return evolve_rows(params, r, points, nullptr, 0, steps, step, stepper, dirs, samples, box, table, status,
                       workspace, workspace_bytes, stream);
}

size_t nlo_bk_vegas_state_doubles(int32_t points, int32_t bins)
{
    if (points < 1 || bins < 2 || bins > 256) return 0;
    return (size_t)points * bk_vegas_state_doubles(bins);
}

static bool check_vegas(const nlo_bk_vegas_options* o, std::string& why)
{
    if (!o) { why = "Vegas options are NULL"; return false; }
    if (o->samples_per_iteration < 2) { why = "Vegas requires at least two samples per iteration"; return false; }
    if (o->warmup_samples == 1 || o->warmup_samples < 0) { why = "warmup_samples must be zero or at least two"; return false; }
    if (o->max_iterations < 1) { why = "Vegas requires at least one iteration"; return false; }
    if (o->min_iterations < 1 || o->min_iterations > o->max_iterations) {
        why = "min_iterations must lie between one and max_iterations";
        return false;
    }
    if (o->bins < 2 || o->bins > 256) { why = "bins must be 2..256"; return false; }
    if (!(o->reuse_warmup_fraction >= 0.0 && o->reuse_warmup_fraction <= 1.0)) {
        why = "reuse_warmup_fraction must lie between zero and one";
        return false;
    }
    if (!(o->epsrel >= 0.0) || !(o->epsabs >= 0.0)) { why = "epsrel and epsabs must be non-negative"; return false; }
    if (o->replicas < 0 || o->replicas > 16) { why = "replicas must be 0..16"; return false; }
    if (o->warmup_samples + (int64_t)o->max_iterations * o->samples_per_iteration > (int64_t(1) << 30)) {
        why = "the Vegas rounds of one right-hand side exceed 2^30 Sobol points";
        return false;
    }
    return true;
}

size_t nlo_bk_vegas_workspace_bytes(int32_t points, const nlo_bk_vegas_options* options)
{
    std::string why;
    if (points < 3 || !check_vegas(options, why)) return 0;
    return nlo_bk_rhs_workspace_bytes(points) + align_up(bk_vegas_scratch_bytes(points, options->bins));
}

// The Vegas buffers at the end of the workspace (after the right-hand side and stage rows);
// the replicas' direction sets stay in `replica_dirs` for the call.
static BkVegasCall vegas_call(void* workspace, int points, const nlo_bk_vegas_options* options, double* state,
                              const nlo_sobol_dirs* dirs, std::vector<SobolDirsArg>& replica_dirs)
{
    char* scratch = static_cast<char*>(workspace) + nlo_bk_rhs_workspace_bytes(points);
    BkVegasCall call = bk_vegas_carve(scratch, points, *options, state);
    replica_dirs.clear();
    for (int k = 0; k < options->replicas; ++k) replica_dirs.push_back(to_arg(dirs + 1 + k));
    call.replica_dirs = replica_dirs.data();
    return call;
}

static bool check_vegas_dirs(const nlo_sobol_dirs* dirs, const nlo_bk_vegas_options* o, std::string& why)
{
    for (int k = 0; k <= o->replicas; ++k)
        if (!check_dirs(dirs + k, 4, why)) {
            why = "dirs[" + std::to_string(k) + "]: " + why;
            return false;
        }
    return true;
}

int nlo_bk_rhs_vegas(const nlo_bk_params* params, const double* r, int32_t points, const double* hist_y,
                     const double* hist_N, int32_t rows, int32_t shard, int32_t shards,
                     const nlo_bk_vegas_options* options, const nlo_sobol_dirs* dirs, const nlo_bk_box* box,
                     double* state, double* dndy, double* k1, double* k2kf, void* workspace, size_t workspace_bytes,
                     void* stream)
{
    std::string why;
    if (!check_params(params, why)) return fail(NLO_ERR_INVALID, why);
    if (!check_dirs(dirs, 4, why)) return fail(NLO_ERR_INVALID, why);
    if (!check_vegas(options, why)) return fail(NLO_ERR_INVALID, why);
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "points must be 3..4096");
    if (rows < 1) return fail(NLO_ERR_INVALID, "the history needs at least one row");
    if (shards < 1 || shard < 0 || shard >= shards) return fail(NLO_ERR_INVALID, "shard must lie in [0, shards)");
    if (params->kinematical_constraint && !hist_y)
        return fail(NLO_ERR_INVALID, "the kinematical constraint needs the history rapidities");
    if (!r || !hist_N || !dndy || !box || !state) return fail(NLO_ERR_INVALID, "NULL buffer");
    if (!workspace || workspace_bytes < nlo_bk_vegas_workspace_bytes(points, options))
        return fail(NLO_ERR_WORKSPACE, "workspace too small for nlo_bk_rhs_vegas");
    if (!check_vegas_dirs(dirs, options, why)) return fail(NLO_ERR_INVALID, why);
    const RhsBuffers b = carve(workspace, points);
    std::vector<SobolDirsArg> replica_dirs;
    const BkVegasCall call = vegas_call(workspace, points, options, state, dirs, replica_dirs);
    const double* N = hist_N + (size_t)(rows - 1) * points;
    const SideStream side;
    return run_rhs(*params, r, N, points, to_arg(dirs), (uint64_t)options->samples_per_iteration, *box, dndy, k1, k2kf,
                   b, false, (cudaStream_t)stream, shard, shards, hist_y, hist_N, rows, &side, &call);
}

int nlo_bk_evolve_vegas(const nlo_bk_params* params, const double* r, int32_t points, const double* y, int32_t first,
                        int32_t steps, double step, int32_t stepper, const nlo_bk_vegas_options* options,
                        const nlo_sobol_dirs* dirs, const nlo_bk_box* box, double* state, double* table,
                        uint32_t* status, void* workspace, size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!check_vegas(options, why)) return fail(NLO_ERR_INVALID, why);
    if (!state) return fail(NLO_ERR_INVALID, "NULL buffer");
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "points must be 3..4096");
    if (!workspace || workspace_bytes < nlo_bk_vegas_workspace_bytes(points, options))
        return fail(NLO_ERR_WORKSPACE, "workspace too small for nlo_bk_evolve_vegas");
    if (!dirs) return fail(NLO_ERR_INVALID, "dirs is NULL");
    if (!check_vegas_dirs(dirs, options, why)) return fail(NLO_ERR_INVALID, why);
    std::vector<SobolDirsArg> replica_dirs;
    const BkVegasCall call = vegas_call(workspace, points, options, state, dirs, replica_dirs);
    return evolve_rows(params, r, points, y, first, steps, step, stepper, dirs, options->samples_per_iteration, box,
                       table, status, workspace, workspace_bytes, stream, &call);
}

size_t nlo_bk_sets_workspace_bytes(int32_t points, int32_t sets, int32_t waves)
{
    if (points < 3 || points > 4096 || sets < 1 || sets > kMaxSets || waves < 1 || waves > 64) return 0;
    return sets_bytes(points, sets, sets_layout(points, sets, waves), nullptr);
}

int nlo_bk_evolve_sets(const nlo_bk_params* params, const double* r, int32_t points, int32_t sets,
                       double* const* tables, int32_t steps, double step, int32_t stepper,
                       const nlo_sobol_dirs* dirs, const int64_t* samples, const nlo_bk_box* box, int32_t waves,
                       uint32_t* status, void* workspace, size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!check_params(params, why)) return fail(NLO_ERR_INVALID, why);
    if (params->kinematical_constraint)
        return fail(NLO_ERR_INVALID, "the kinematical constraint is not available for parameter sets");
    if (points < 3 || points > 4096) return fail(NLO_ERR_INVALID, "points must be 3..4096");
    if (sets < 1 || sets > kMaxSets) return fail(NLO_ERR_INVALID, "sets must be 1..256");
    if (!dirs) return fail(NLO_ERR_INVALID, "dirs is NULL");
    for (int i = 0; i < sets; ++i)
        if (!check_dirs(dirs + i, 4, why)) return fail(NLO_ERR_INVALID, "set " + std::to_string(i) + ": " + why);
    if (waves < 1 || waves > 64) return fail(NLO_ERR_INVALID, "waves must be 1..64");
    if (steps < 0) return fail(NLO_ERR_INVALID, "steps must be non-negative");
    if (!(step > 0) || !std::isfinite(step)) return fail(NLO_ERR_INVALID, "step must be positive");
    if (stepper != NLO_STEPPER_EULER && stepper != NLO_STEPPER_RK3 && stepper != NLO_STEPPER_RK4)
        return fail(NLO_ERR_INVALID, "unknown stepper");
    if (!r || !tables || !samples || !status || !box) return fail(NLO_ERR_INVALID, "NULL buffer");
    for (int i = 0; i < sets; ++i) {
        if (!tables[i]) return fail(NLO_ERR_INVALID, "NULL table");
        if (samples[i] < 0 || samples[i] > (int64_t(1) << 30)) return fail(NLO_ERR_INVALID, "samples out of range");
    }
    const SetsLayout L = sets_layout(points, sets, waves);
    if (!workspace || workspace_bytes < sets_bytes(points, sets, L, nullptr))
        return fail(NLO_ERR_WORKSPACE, "workspace too small for nlo_bk_evolve_sets");
    cudaStream_t s = (cudaStream_t)stream;
    size_t off[9];
    sets_bytes(points, sets, L, off);
    char* base = static_cast<char*>(workspace);
    double* spline = reinterpret_cast<double*>(base + off[0]);
    double* factor = reinterpret_cast<double*>(base + off[1]);
    int32_t* active = reinterpret_cast<int32_t*>(base + off[2]);
    int32_t* counts = reinterpret_cast<int32_t*>(base + off[3]);
    double* k1 = reinterpret_cast<double*>(base + off[4]);
    double* k2kf = reinterpret_cast<double*>(base + off[5]);
    double* partial = reinterpret_cast<double*>(base + off[6]);
    double* stage = reinterpret_cast<double*>(base + off[7]);
    SetTable* table = reinterpret_cast<SetTable*>(base + off[8]);
    const size_t S = (size_t)sets, n = (size_t)points;
    double* kk[4] = {stage, stage + S * n, stage + 2 * S * n, stage + 3 * S * n};
    double* tmp = stage + 4 * S * n;
    double* cur = stage + 5 * S * n;

    // slots in order of decreasing budget (ties by set index), so that slot 0 of every group
    // holds the group's largest budget and sets of one budget share CTAs
    int32_t order[kMaxSets];
    for (int i = 0; i < sets; ++i) order[i] = i;
    std::stable_sort(order, order + sets, [&](int32_t a, int32_t b) { return samples[a] > samples[b]; });
    const int slots = L.groups * L.per_cta;
    int32_t slot_set[kMaxSlots];
    for (int q = 0; q < slots; ++q) slot_set[q] = q < sets ? order[q] : -1;
    const bool nlo = order_has_nlo(params->order);
    std::vector<SobolDirsArg> set_dirs(sets);
    const SobolDirsArg* dir_ptrs[kMaxSets];
    for (int i = 0; i < sets; ++i) {
        set_dirs[i] = to_arg(dirs + i);
        dir_ptrs[i] = &set_dirs[i];
    }
    cudaError_t e = launch_sets_setup(tables, samples, slot_set, dir_ptrs, sets, slots, nlo, table, s);
    if (e != cudaSuccess) return cuda_fail(e, "sets setup");
    if ((e = cudaMemsetAsync(status, 0, sizeof(uint32_t) * S, s)) != cudaSuccess) return cuda_fail(e, "status reset");
    double* const* rows = reinterpret_cast<double* const*>(base + off[8] + offsetof(SetTable, rows));
    RowsArg work, fixed;
    work.base = tmp;
    work.stride = n;
    fixed.base = cur;
    fixed.stride = n;
    const int clamp = params->force_positive ? 1 : 0;
    const SideStream side;
    bool factor_ready = false;
    // as in evolve_rows: the first step launches its kernels one by one, the later ones
    // replay a recording of one step that advances the fixed rows in place
    StepGraph graph;
    bool recorded = false;
    auto step_from = [&](const RowsArg& now, const RowsArg& next, cudaStream_t s) {
        auto rhs = [&](int src, int k) {
            const RowsArg& in = src < 0 ? now : work;
            if ((e = launch_splines(r, in, points, sets, params->force_positive, factor, factor_ready ? 0 : 1, spline,
                                    s)) != cudaSuccess)
                return cuda_fail(e, "splines");
            factor_ready = true;
            if ((e = launch_active(in, points, sets, 0, 1, active, counts, s)) != cudaSuccess)
                return cuda_fail(e, "active");
            const bool beside = side.ok;
            cudaStream_t k1_stream = beside ? side.aux : s;
            if (beside && ((e = cudaEventRecord(side.fork, s)) != cudaSuccess ||
                           (e = cudaStreamWaitEvent(side.aux, side.fork, 0)) != cudaSuccess))
                return cuda_fail(e, "fork");
            if ((e = launch_k1(*params, r, points, spline, active, counts, k1, k1_stream, K1History(), sets)) !=
                cudaSuccess)
                return cuda_fail(e, "k1");
            if (beside && (e = cudaEventRecord(side.join, side.aux)) != cudaSuccess) return cuda_fail(e, "join");
            if (nlo) {
                if ((e = launch_k2kf_sets(*params, r, points, sets, spline, spline_doubles(points), active, counts,
                                          *box, L, table, k2kf, partial, s)) != cudaSuccess)
                    return cuda_fail(e, "k2kf sets");
            } else if ((e = cudaMemsetAsync(k2kf, 0, sizeof(double) * 3 * S * n, s)) != cudaSuccess) {
                return cuda_fail(e, "k2kf clear");
            }
            if (beside && (e = cudaStreamWaitEvent(s, side.join, 0)) != cudaSuccess) return cuda_fail(e, "join");
            if ((e = launch_assemble_sets(k1, k2kf, points, sets, table, kk[k], s)) != cudaSuccess)
                return cuda_fail(e, "assemble");
            return (int)NLO_OK;
        };
        auto comb = [&](int nk, const int* ks, const double* coef, int dst) {
            const double* kp[4];
            for (int j = 0; j < nk; ++j) kp[j] = kk[ks[j]];
            const cudaError_t err = launch_axpy_sets(now, kp, coef, nk, points, sets, dst ? next : work,
                                                     dst ? clamp : 0, dst ? status : nullptr, s);
            return err == cudaSuccess ? (int)NLO_OK : cuda_fail(err, "stage");
        };
        return step_sequence(stepper, step, rhs, comb);
    };
    for (int it = 0; it < steps; ++it) {
        RowsArg now, next;
        now.ptrs = rows;
        now.offset = (size_t)it * n;
        next.ptrs = rows;
        next.offset = (size_t)(it + 1) * n;
        if (it == 1 && replay_pays(points)) {
            recorded = graph.capture([&](cudaStream_t st) { return step_from(fixed, fixed, st); });
            // a combination without terms copies the rows
            if (recorded &&
                (e = launch_axpy_sets(now, nullptr, nullptr, 0, points, sets, fixed, 0, nullptr, s)) != cudaSuccess)
                return cuda_fail(e, "step rows");
        }
        if (recorded) {
            if ((e = cudaGraphLaunch(graph.exec, s)) != cudaSuccess) return cuda_fail(e, "step graph");
            if ((e = launch_axpy_sets(fixed, nullptr, nullptr, 0, points, sets, next, 0, nullptr, s)) != cudaSuccess)
                return cuda_fail(e, "step rows");
            continue;
        }
        const int rc = step_from(now, next, s);
        if (rc != NLO_OK) return rc;
    }
    return NLO_OK;
}

int nlo_bk_evolve_history(const nlo_bk_params* params, const double* r, int32_t points, const double* y,
                          int32_t first, int32_t steps, double step, int32_t stepper, const nlo_sobol_dirs* dirs,
                          int64_t samples, const nlo_bk_box* box, double* table, uint32_t* status, void* workspace,
                          size_t workspace_bytes, void* stream)
{
    if (!y) return fail(NLO_ERR_INVALID, "NULL buffer");
    return evolve_rows(params, r, points, y, first, steps, step, stepper, dirs, samples, box, table, status,
                       workspace, workspace_bytes, stream);
}

}  // extern "C"
