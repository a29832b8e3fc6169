// extern "C" entry points of the NLO DIS path (declared in include/nlo_b200.h): argument
// checks, conversion of the job descriptions into device argument blocks inside the
// caller's workspace, and the Vegas round sequence.  Nothing here allocates device memory
// and nothing synchronises the stream: argument blocks go up with cudaMemcpyAsync from
// host staging vectors (pageable host-to-device copies are staged before the call returns).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dis_internal.h"
#include "dis_terms.cuh"

namespace nlo {
namespace {

using dis::DisArgs;
using dis::InnerRule;

int dfail(int code, const std::string& message) { return set_last_error(code, message.c_str()); }

int dcuda(cudaError_t e, const char* where)
{
    return dfail(NLO_ERR_CUDA, std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

bool check_kin(const nlo_dis_kinematics& k, int term, std::string& why)
{
    if (!(k.Q2 > 0) || !std::isfinite(k.Q2)) { why = "Q2 must be positive and finite"; return false; }
    if (!(k.xbj > 0 && k.xbj <= 1)) { why = "x_Bj must lie in (0, 1]"; return false; }
    if (!(k.maxr > 0)) { why = "maxr must be positive"; return false; }
    if (!(k.c2_alpha > 0) || !(k.max_alpha > 0)) { why = "C2_alpha and the freeze value must be positive"; return false; }
    if (term == dis::kTermLO) {
        if (k.n_quarks < 1 || k.n_quarks > NLO_DIS_MAX_QUARKS) { why = "LO needs 1..8 quarks"; return false; }
        for (int q = 0; q < k.n_quarks; ++q)
            if (!(k.lo_mass[q] >= 0)) { why = "quark masses must be non-negative"; return false; }
    } else if (!(k.mf > 0)) {
        why = "the NLO terms need a positive quark mass";
        return false;
    }
    return true;
}

bool check_dipole(const nlo_dipole* d, std::string& why)
{
    if (!d) { why = "dipole is NULL"; return false; }
    if (d->kind == NLO_DIPOLE_GBW) {
        if (!(d->qs0sqr > 0) || !(d->x0 > 0)) { why = "GBW needs Qs0sqr > 0 and x0 > 0"; return false; }
        return true;
    }
    if (d->kind == NLO_DIPOLE_TABLE) {
        if (!d->table) { why = "table dipole without a prepared table"; return false; }
        if (d->nr < 9 || d->ny < 1) { why = "BK table needs nr >= 9 and ny >= 1"; return false; }
        return true;
    }
    why = "unknown dipole kind";
    return false;
}

template <typename T>
DisArgs<T> make_args(const nlo_dis_kinematics& k, const nlo_dipole& d)
{
    DisArgs<T> a;
    std::memset(&a, 0, sizeof(a));
    a.Q2 = k.Q2;
    a.xbj = k.xbj;
    a.mf = k.mf;
    a.maxr = k.maxr;
    // evolution_rapidity_dipole (dis/observables.py:62-76)
    const double W2d = (1.0 - k.xbj) * k.Q2 / k.xbj;
    const double X = k.mass_dependent_x ? (k.Q2 + 4.0 * k.mf * k.mf) / (k.Q2 + W2d) : k.Q2 / (k.Q2 + W2d);
    a.Ydip = std::log(1.0 / X);
    const double X0 = d.kind == NLO_DIPOLE_GBW ? d.x0 : 1.0;  // dipole.X0()
    a.Ylo = std::fmax(std::log(X0 / k.xbj), 0.0);
    a.W2 = k.Q2 / k.xbj;  // evolution_rapidity_qqg, z2_lower_bound (:56-85)
    a.z2min = dis::kQ0sqr / a.W2;
    a.gm1 = 4.0 * k.mf * k.mf / k.Q2 / (1.0 + std::sqrt(1.0 + 4.0 * k.mf * k.mf / k.Q2));
    a.n_quarks = k.n_quarks;
    for (int q = 0; q < dis::kMaxQuarks; ++q) {
        a.lo_mass[q] = k.lo_mass[q];
        a.lo_e2[q] = k.lo_charge2[q];
    }
    a.transverse = k.transverse != 0;
    a.finite_nc = k.finite_nc != 0;
    a.parent_coupling = k.parent_coupling != 0;
    a.coup.b0 = (T)((11.0 * dis::kNc - 2.0 * k.active_flavors) / (12.0 * dis::kPi));
    a.coup.log_scale = (T)std::log(4.0 * k.c2_alpha / (dis::kLambdaQCD * dis::kLambdaQCD));
    a.coup.max_alpha = (T)k.max_alpha;
    a.coup.smooth_left = (T)(2.0 / 0.2 * std::log(2.5));
    a.coup.smooth = k.smooth_coupling != 0;
    a.table = d.kind == NLO_DIPOLE_TABLE;
    if (a.table) {
        a.tab = dis::table_view(d.table, d.nr, d.ny);
    } else {
        a.gbw.qs0sqr = (T)d.qs0sqr;
        a.gbw.lambda = (T)d.lambda;
        a.gbw.gamma = (T)d.gamma;
        a.gbw.y0 = (T)std::log(1.0 / d.x0);
        a.gbw_min_r = 1e-30;
        a.gbw_max_r = 1e3;
    }
    return a;
}

bool make_rule(int term, int points, InnerRule& rule, std::string& why)
{
    std::memset(&rule, 0, sizeof(rule));
    if (term != dis::kTermI2N && term != dis::kTermI3N) return true;
    if (points < 8 || points > dis::kMaxInner) { why = "the inner rule needs 8..128 points"; return false; }
    std::vector<double> x(points), w(points);
    gauss_legendre_rule(points, x.data(), w.data());
    rule.n = points;
    for (int i = 0; i < points; ++i) {
        // y = t^3, t = (node + 1)/2, weight w/2 * 3 t^2 (custom_kernels/dis/i2_i3/extension.py:21-35)
        const double t = 0.5 * (x[i] + 1.0);
        rule.y[i] = t * t * t;
        rule.w[i] = 0.5 * w[i] * 3.0 * t * t;
    }
    return true;
}

constexpr size_t kAlign = 256;
size_t align_up(size_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }
size_t args_bytes(int jobs) { return align_up((size_t)jobs * std::max(sizeof(DisArgs<double>), sizeof(DisArgs<float>))); }

// Argument blocks of `jobs` jobs; job j takes the dipole dipoles[j * dipole_stride]
// (stride 0: one dipole for every job).
int upload_args(const nlo_dis_kinematics* kin, int jobs, const nlo_dipole* dipoles, int dipole_stride, int precision,
                void* dst, cudaStream_t stream)
{
    cudaError_t e;
    if (precision == NLO_PRECISION_FP64) {
        std::vector<DisArgs<double>> h(jobs);
        for (int j = 0; j < jobs; ++j) h[j] = make_args<double>(kin[j], dipoles[(size_t)j * dipole_stride]);
        e = cudaMemcpyAsync(dst, h.data(), sizeof(DisArgs<double>) * jobs, cudaMemcpyHostToDevice, stream);
    } else {
        std::vector<DisArgs<float>> h(jobs);
        for (int j = 0; j < jobs; ++j) h[j] = make_args<float>(kin[j], dipoles[(size_t)j * dipole_stride]);
        e = cudaMemcpyAsync(dst, h.data(), sizeof(DisArgs<float>) * jobs, cudaMemcpyHostToDevice, stream);
    }
    return e == cudaSuccess ? NLO_OK : dcuda(e, "DIS argument upload");
}

int sm_count()
{
    static int sms = [] {
        int device = 0, n = 148;
        if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
        return n > 0 ? n : 148;
    }();
    return sms;
}

// CTAs per job per round: one sample per thread at most, and over all jobs about four
// times the resident capacity (three 256-thread CTAs per SM), so that CTAs of uneven cost
// even out (a fixed function of the job count, the sample count and the SM count)
int vegas_blocks(int64_t samples, int jobs)
{
    const int64_t by_samples = (samples + dis::kVegasThreads - 1) / dis::kVegasThreads;
    const int64_t want = (4 * 3 * (int64_t)sm_count() + jobs - 1) / jobs;
    int64_t b = std::min(by_samples, want);
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 65535));
}

size_t state_doubles(int term, int bins) { return (size_t)dis::term_dims(term) * (bins + 1) + dis::kStSlots; }

struct VegasCarve {
    size_t args, dirs, partial, reduced, counts, total;
};

VegasCarve vegas_carve(int jobs, int term, const nlo_vegas_options& o)
{
    const int D = dis::term_dims(term);
    const int64_t most = std::max<int64_t>(o.samples_per_iteration, o.warmup_samples);
    const int blocks = vegas_blocks(most, jobs);
    VegasCarve c;
    c.args = 0;
    c.dirs = align_up(c.args + args_bytes(jobs));
    c.partial = align_up(c.dirs + sizeof(SobolDirsArg) * (size_t)jobs);
    c.reduced = align_up(c.partial + sizeof(double) * (size_t)jobs * blocks * (2 + (size_t)D * o.bins));
    c.counts = align_up(c.reduced + sizeof(double) * (size_t)jobs * (2 + (size_t)D * o.bins));
    c.total = align_up(c.counts + sizeof(int32_t) * (size_t)jobs * (size_t)D * o.bins);
    return c;
}

bool check_options(const nlo_vegas_options* o, int term, std::string& why)
{
    if (!o) { why = "options is NULL"; return false; }
    if (o->bins < 2 || o->bins > dis::kMaxBins) { why = "bins must lie in 2..256"; return false; }
    if (o->max_iterations < 1 || o->min_iterations < 1 || o->min_iterations > o->max_iterations) {
        why = "min_iterations must lie between one and max_iterations";
        return false;
    }
    if (o->samples_per_iteration < 2) { why = "Vegas requires at least two samples"; return false; }
    if (o->warmup_samples == 1 || o->warmup_samples < 0) { why = "warmup_samples must be zero or at least two"; return false; }
    const int64_t total = o->samples_per_iteration * (int64_t)o->max_iterations + o->warmup_samples;
    if (total > (int64_t(1) << 30)) { why = "Sobol index range exceeds 2^30"; return false; }
    if (o->precision != NLO_PRECISION_MIXED && o->precision != NLO_PRECISION_FP64) { why = "unknown precision"; return false; }
    if (!(o->epsrel >= 0) || !(o->epsabs >= 0)) { why = "tolerances must be non-negative"; return false; }
    (void)term;
    return true;
}

}  // namespace
}  // namespace nlo

using namespace nlo;

extern "C" {

size_t nlo_dis_table_doubles(int32_t nr, int32_t ny) { return nr < 2 || ny < 1 ? 0 : dis::table_doubles(nr, ny); }

int nlo_dis_table_prepare_interpolated(const double* r, const double* y, const double* N, int32_t nr, int32_t ny,
                                       double x0, int32_t interpolation, double* table, void* stream)
{
    if (!r || !y || !N || !table) return dfail(NLO_ERR_INVALID, "nlo_dis_table_prepare: NULL argument");
    if (nr < 9 || ny < 1) return dfail(NLO_ERR_INVALID, "BKDipole requires at least nine r points and one rapidity");
    if (!(x0 > 0) || !std::isfinite(x0)) return dfail(NLO_ERR_INVALID, "x0 must be positive and finite");
    if (interpolation != NLO_INTERP_SPLINE_LINEAR && interpolation != NLO_INTERP_LINEAR_LINEAR)
        return dfail(NLO_ERR_INVALID, "unknown table interpolation");
    const double y0 = std::fmax(0.0, std::log(1.0 / x0));
    cudaError_t e = dis_launch_table_prepare(r, y, N, nr, ny, y0, interpolation, table,
                                             static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? NLO_OK : dcuda(e, "table prepare launch");
}

int nlo_dis_table_prepare(const double* r, const double* y, const double* N, int32_t nr, int32_t ny, double x0,
                          double* table, void* stream)
{
    return nlo_dis_table_prepare_interpolated(r, y, N, nr, ny, x0, NLO_INTERP_SPLINE_LINEAR, table, stream);
}

int nlo_dis_table_initialize(double* table, int32_t nr, int32_t ny, double Y, void* stream)
{
    if (!table || nr < 9 || ny < 1) return dfail(NLO_ERR_INVALID, "nlo_dis_table_initialize: bad table");
    if (!(Y >= 0) || !std::isfinite(Y)) return dfail(NLO_ERR_INVALID, "cannot initialize interpolation at negative Y");
    if ((size_t)nr * 3 * sizeof(double) > 200 * 1024) return dfail(NLO_ERR_INVALID, "table longer than 8533 r points");
    cudaError_t e = dis_launch_table_initialize(table, nr, ny, Y, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? NLO_OK : dcuda(e, "table initialize launch");
}

int nlo_dis_integrand(const nlo_dis_kinematics* kin, int32_t term, const nlo_dipole* dipole, int32_t inner_points,
                      int32_t precision, const double* x, int64_t n, double* out, void* stream)
{
    std::string why;
    if (!kin || !x || !out) return dfail(NLO_ERR_INVALID, "nlo_dis_integrand: NULL argument");
    if (term < 0 || term >= dis::kTermCount) return dfail(NLO_ERR_INVALID, "unknown DIS term");
    if (precision != NLO_PRECISION_MIXED && precision != NLO_PRECISION_FP64) return dfail(NLO_ERR_INVALID, "unknown precision");
    if (!check_kin(*kin, term, why) || !check_dipole(dipole, why)) return dfail(NLO_ERR_INVALID, why);
    if (n < 0) return dfail(NLO_ERR_INVALID, "negative point count");
    InnerRule rule;
    if (!make_rule(term, inner_points, rule, why)) return dfail(NLO_ERR_INVALID, why);
    if (n == 0) return NLO_OK;
    cudaError_t e;
    if (precision == NLO_PRECISION_FP64) {
        const DisArgs<double> a = make_args<double>(*kin, *dipole);
        e = dis_launch_points(precision, term, &a, rule, x, n, out, static_cast<cudaStream_t>(stream));
    } else {
        const DisArgs<float> a = make_args<float>(*kin, *dipole);
        e = dis_launch_points(precision, term, &a, rule, x, n, out, static_cast<cudaStream_t>(stream));
    }
    return e == cudaSuccess ? NLO_OK : dcuda(e, "DIS integrand launch");
}

int nlo_dis_dipole_amplitude(const nlo_dipole* dipole, const double* r, const double* Y, int64_t n, int32_t precision,
                             double* out, void* stream)
{
    std::string why;
    if (!r || !Y || !out) return dfail(NLO_ERR_INVALID, "nlo_dis_dipole_amplitude: NULL argument");
    if (!check_dipole(dipole, why)) return dfail(NLO_ERR_INVALID, why);
    if (precision != NLO_PRECISION_MIXED && precision != NLO_PRECISION_FP64) return dfail(NLO_ERR_INVALID, "unknown precision");
    if (n < 0) return dfail(NLO_ERR_INVALID, "negative point count");
    if (n == 0) return NLO_OK;
    nlo_dis_kinematics k;
    std::memset(&k, 0, sizeof(k));
    k.Q2 = 1.0;
    k.xbj = 1.0;
    k.c2_alpha = 1.0;
    k.max_alpha = 1.0;
    cudaError_t e;
    if (precision == NLO_PRECISION_FP64) {
        const DisArgs<double> a = make_args<double>(k, *dipole);
        e = dis_launch_amplitude(precision, &a, r, Y, n, out, static_cast<cudaStream_t>(stream));
    } else {
        const DisArgs<float> a = make_args<float>(k, *dipole);
        e = dis_launch_amplitude(precision, &a, r, Y, n, out, static_cast<cudaStream_t>(stream));
    }
    return e == cudaSuccess ? NLO_OK : dcuda(e, "dipole amplitude launch");
}

size_t nlo_dis_gauss_legendre_workspace_bytes(int32_t jobs) { return jobs < 1 ? 0 : args_bytes(jobs); }

static int gauss_legendre_jobs(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term, const nlo_dipole* dipoles,
                               int dipole_stride, int32_t points, int32_t precision, double* out, void* workspace,
                               size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!kin || !out || !dipoles) return dfail(NLO_ERR_INVALID, "nlo_dis_gauss_legendre: NULL argument");
    if (jobs < 1) return dfail(NLO_ERR_INVALID, "jobs must be positive");
    if (term != dis::kTermLO && term != dis::kTermDip0) return dfail(NLO_ERR_INVALID, "the tensor rule serves the 2D terms");
    if (points < 4 || points > 64) return dfail(NLO_ERR_INVALID, "points must lie in 4..64");
    if (precision != NLO_PRECISION_MIXED && precision != NLO_PRECISION_FP64) return dfail(NLO_ERR_INVALID, "unknown precision");
    for (int j = 0; j < jobs; ++j) {
        if (!check_dipole(&dipoles[(size_t)j * dipole_stride], why)) return dfail(NLO_ERR_INVALID, why);
        if (!check_kin(kin[j], term, why)) return dfail(NLO_ERR_INVALID, why);
    }
    if (!workspace || workspace_bytes < args_bytes(jobs)) return dfail(NLO_ERR_WORKSPACE, "workspace missing or too small");
    dis::GLRules gl;
    std::memset(&gl, 0, sizeof(gl));
    gl.n_fine = points;
    gl.n_coarse = std::max(2, points / 2);
    std::vector<double> x(points), w(points);
    gauss_legendre_rule(points, x.data(), w.data());
    for (int i = 0; i < points; ++i) {
        gl.x_fine[i] = 0.5 * (x[i] + 1.0);
        gl.w_fine[i] = 0.5 * w[i];
    }
    gauss_legendre_rule(gl.n_coarse, x.data(), w.data());
    for (int i = 0; i < gl.n_coarse; ++i) {
        gl.x_coarse[i] = 0.5 * (x[i] + 1.0);
        gl.w_coarse[i] = 0.5 * w[i];
    }
    InnerRule rule;
    make_rule(term, 48, rule, why);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = upload_args(kin, jobs, dipoles, dipole_stride, precision, workspace, s);
    if (rc != NLO_OK) return rc;
    cudaError_t e = dis_launch_gl(precision, term, workspace, jobs, rule, gl, out, s);
    return e == cudaSuccess ? NLO_OK : dcuda(e, "DIS Gauss-Legendre launch");
}

int nlo_dis_gauss_legendre(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term, const nlo_dipole* dipole,
                           int32_t points, int32_t precision, double* out, void* workspace, size_t workspace_bytes,
                           void* stream)
{
    return gauss_legendre_jobs(kin, jobs, term, dipole, 0, points, precision, out, workspace, workspace_bytes, stream);
}

int nlo_dis_gauss_legendre_dipoles(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term,
                                   const nlo_dipole* dipoles, int32_t points, int32_t precision, double* out,
                                   void* workspace, size_t workspace_bytes, void* stream)
{
    return gauss_legendre_jobs(kin, jobs, term, dipoles, 1, points, precision, out, workspace, workspace_bytes, stream);
}

size_t nlo_dis_vegas_state_doubles(int32_t term, int32_t bins)
{
    if (term < 0 || term >= dis::kTermCount || bins < 2) return 0;
    return state_doubles(term, bins);
}

size_t nlo_dis_vegas_workspace_bytes(int32_t jobs, int32_t term, const nlo_vegas_options* options)
{
    std::string why;
    if (jobs < 1 || term < 0 || term >= dis::kTermCount || !check_options(options, term, why)) return 0;
    return vegas_carve(jobs, term, *options).total;
}

static int vegas_jobs(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term, const nlo_dipole* dipoles,
                      int dipole_stride, const nlo_vegas_options* options, const nlo_sobol_dirs* dirs, double* state,
                      void* workspace, size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!kin || !dirs || !state || !dipoles) return dfail(NLO_ERR_INVALID, "nlo_dis_vegas: NULL argument");
    if (jobs < 1) return dfail(NLO_ERR_INVALID, "jobs must be positive");
    if (term < 0 || term >= dis::kTermCount) return dfail(NLO_ERR_INVALID, "unknown DIS term");
    if (!check_options(options, term, why)) return dfail(NLO_ERR_INVALID, why);
    const int D = dis::term_dims(term);
    for (int j = 0; j < jobs; ++j) {
        if (!check_dipole(&dipoles[(size_t)j * dipole_stride], why)) return dfail(NLO_ERR_INVALID, why);
        if (!check_kin(kin[j], term, why)) return dfail(NLO_ERR_INVALID, why);
        if (dirs[j].dims < D || dirs[j].dims > 8) return dfail(NLO_ERR_INVALID, "Sobol dimension count does not match the term");
    }
    InnerRule rule;
    if (!make_rule(term, options->inner_points, rule, why)) return dfail(NLO_ERR_INVALID, why);
    const VegasCarve c = vegas_carve(jobs, term, *options);
    if (!workspace || workspace_bytes < c.total) return dfail(NLO_ERR_WORKSPACE, "workspace missing or too small");
    unsigned char* ws = static_cast<unsigned char*>(workspace);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = upload_args(kin, jobs, dipoles, dipole_stride, options->precision, ws + c.args, s);
    if (rc != NLO_OK) return rc;
    static_assert(sizeof(SobolDirsArg) == sizeof(nlo_sobol_dirs), "Sobol direction layouts differ");
    cudaError_t e = cudaMemcpyAsync(ws + c.dirs, dirs, sizeof(nlo_sobol_dirs) * (size_t)jobs, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return dcuda(e, "Sobol direction upload");
    const int stride = (int)state_doubles(term, options->bins);
    int32_t* counts = reinterpret_cast<int32_t*>(ws + c.counts);
    e = dis_launch_vegas_init(state, stride, D, options->bins, jobs, options->keep_edges, counts, s);
    if (e != cudaSuccess) return dcuda(e, "Vegas init launch");
    dis::VegasLaunch L;
    L.args = ws + c.args;
    L.dirs = reinterpret_cast<const SobolDirsArg*>(ws + c.dirs);
    L.rule = &rule;
    L.state = state;
    L.state_stride = stride;
    L.jobs = jobs;
    L.bins = options->bins;
    L.partial = reinterpret_cast<double*>(ws + c.partial);
    L.reduced = reinterpret_cast<double*>(ws + c.reduced);
    L.counts = counts;
    L.min_iterations = options->min_iterations;
    L.epsrel = options->epsrel;
    L.epsabs = options->epsabs;
    uint64_t offset = 0;
    const int rounds = options->max_iterations + (options->warmup_samples > 0 ? 1 : 0);
    for (int it = 0; it < rounds; ++it) {
        const bool warm = options->warmup_samples > 0 && it == 0;
        L.samples = (uint64_t)(warm ? options->warmup_samples : options->samples_per_iteration);
        L.offset = offset;
        L.warmup = warm ? 1 : 0;
        L.blocks_per_job = vegas_blocks((int64_t)L.samples, jobs);
        e = dis_launch_vegas_round(options->precision, term, L, s);
        if (e != cudaSuccess) return dcuda(e, "Vegas round launch");
        offset += L.samples;
    }
    return NLO_OK;
}

int nlo_dis_vegas(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term, const nlo_dipole* dipole,
                  const nlo_vegas_options* options, const nlo_sobol_dirs* dirs, double* state, void* workspace,
                  size_t workspace_bytes, void* stream)
{
    return vegas_jobs(kin, jobs, term, dipole, 0, options, dirs, state, workspace, workspace_bytes, stream);
}

int nlo_dis_vegas_dipoles(const nlo_dis_kinematics* kin, int32_t jobs, int32_t term, const nlo_dipole* dipoles,
                          const nlo_vegas_options* options, const nlo_sobol_dirs* dirs, double* state,
                          void* workspace, size_t workspace_bytes, void* stream)
{
    return vegas_jobs(kin, jobs, term, dipoles, 1, options, dirs, state, workspace, workspace_bytes, stream);
}

size_t nlo_dis_fixed_sobol_grid_doubles(int32_t bins)
{
    return bins < 2 ? 0 : (size_t)5 * (bins + 1) + dis::kStSlots;
}

size_t nlo_dis_fixed_sobol_workspace_bytes(const nlo_fixed_sobol_options* options)
{
    std::string why;
    if (!dis_fixed_check(options, why)) return 0;
    return dis_fixed_workspace_bytes(*options);
}

int nlo_dis_fixed_sobol(const nlo_dis_kinematics* kin, const nlo_dipole* dipole, const nlo_fixed_sobol_options* options,
                        const nlo_sobol_dirs* dirs, double* grid, double* estimates, void* workspace,
                        size_t workspace_bytes, void* stream)
{
    std::string why;
    if (!kin || !dirs || !grid || !estimates) return dfail(NLO_ERR_INVALID, "nlo_dis_fixed_sobol: NULL argument");
    if (!dis_fixed_check(options, why) || !check_dipole(dipole, why) || !check_kin(*kin, dis::kTermI1, why))
        return dfail(NLO_ERR_INVALID, why);
    const int rounds = options->training_rounds + options->replicates;
    for (int j = 0; j < rounds; ++j)
        if (dirs[j].dims < 5 || dirs[j].dims > 8) return dfail(NLO_ERR_INVALID, "fixed-Sobol needs 5-dimensional directions");
    const size_t need = dis_fixed_workspace_bytes(*options);
    if (!workspace || workspace_bytes < need) return dfail(NLO_ERR_WORKSPACE, "workspace missing or too small");
    InnerRule rule;
    if (!make_rule(dis::kTermI3N, options->inner_points, rule, why)) return dfail(NLO_ERR_INVALID, why);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(workspace, dirs, sizeof(nlo_sobol_dirs) * (size_t)rounds, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return dcuda(e, "Sobol direction upload");
    if (options->precision == NLO_PRECISION_FP64) {
        const DisArgs<double> a = make_args<double>(*kin, *dipole);
        return dis_run_fixed(options->precision, &a, rule, *options, workspace, grid, estimates, s);
    }
    const DisArgs<float> a = make_args<float>(*kin, *dipole);
    return dis_run_fixed(options->precision, &a, rule, *options, workspace, grid, estimates, s);
}

}  // extern "C"
