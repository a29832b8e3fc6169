// Internal launch interfaces shared by the .cu files of the library.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "../../include/nlo_b200.h"

namespace nlo {

// Sobol direction numbers passed by value as a kernel parameter.
struct SobolDirsArg {
    int dims;
    uint32_t state[8][30];
    uint32_t shift[8];
};

// Gauss-Legendre rules of the fixed K1 integration (8 radial x 24 angular).
struct K1Rule {
    double x8[8], w8[8];
    double x24[24], w24[24];
};

const K1Rule& k1_rule();

// Host checks shared by every entry point that takes BK parameters or Sobol directions:
// false with the reason in `why` when an argument is out of range.
bool check_params(const nlo_bk_params* p, std::string& why);
bool check_dirs(const nlo_sobol_dirs* d, int need, std::string& why);
SobolDirsArg to_arg(const nlo_sobol_dirs* d);

// Buffers of one right-hand-side evaluation carved from the caller's workspace.
struct RhsBuffers {
    double* spline;   // nlo_bk_spline_doubles(points)
    int32_t* active;  // [points]
    int32_t* count;   // [1]
    double* k1;       // [points]
    double* k2kf;     // [points][3]
    double* partial;  // [k2kf_blocks][points][3]
    double* factor;   // [2][points] spline factorisation (grid only)
    double* kc;       // kc_weights_doubles(points): kinematical-constraint window weights
    int32_t* k1_active;  // [points] K1's parents of a shard (sharded right-hand sides)
    int32_t* k1_count;   // [1]
    int k2kf_blocks;
};

__host__ __device__ inline size_t spline_doubles(int points) { return (size_t)points + 8 * (size_t)(points - 1); }
int k2kf_max_blocks();

// Rows of several parameter sets: set s's row is ptrs[s] + offset (rows inside the caller's
// tables) or base + s * stride + offset (rows inside the workspace).
struct RowsArg {
    double* const* ptrs = nullptr;
    double* base = nullptr;
    size_t stride = 0;
    size_t offset = 0;
    __host__ __device__ double* at(int s) const { return (ptrs ? ptrs[s] : base + (size_t)s * stride) + offset; }
};
inline RowsArg single_row(const double* row)
{
    RowsArg a;
    a.base = const_cast<double*>(row);
    return a;
}

// Multi-set K2+Kf (several parameter sets in one launch): a CTA holds `per_cta` set slots of
// `lanes` lanes each; slot q of group g is set slot_set[g * per_cta + q] (-1: empty), and the
// sets are ordered by budget so that slot 0 of a group holds its largest.  CTA row
// blockIdx.y = g * parent_tiles + (parent tile of the set's active list).
constexpr int kMaxSets = 256;
constexpr int kMaxSlots = kMaxSets + 8;  // groups * per_cta (per_cta <= 7)
struct SetsLayout {
    int per_cta = 1, lanes = 64, parent_tiles = 1, groups = 1, threads = 64, blocks = 1;
};
SetsLayout sets_layout(int points, int sets, int waves);
inline size_t sets_partial_doubles(const SetsLayout& L)
{
    return (size_t)L.groups * L.parent_tiles * L.blocks * L.threads * 3;
}
// Per-call set table in the workspace, written by launch_sets_setup.
constexpr int kSetDirsWords = 4 * 30 + 4;  // state[4][30], shift[4]: the K2+Kf box's four dimensions
struct SetTable {
    double* rows[kMaxSets];      // each set's table (row 0 = the initial row)
    uint32_t samples[kMaxSets];  // Sobol budget per set
    int32_t slot_set[kMaxSlots]; // set of each slot, -1 empty
    int32_t set_slot[kMaxSets];  // slot of each set
    double inv[kMaxSets];        // 1 / samples (0 without NLO kernels)
    uint32_t dirs[kMaxSets][kSetDirsWords];  // Sobol directions of dimensions 0..3 and their shifts
};
cudaError_t launch_sets_setup(double* const* rows, const int64_t* samples, const int32_t* slot_set,
                              const SobolDirsArg* const* dirs, int sets, int slots, bool nlo, SetTable* table,
                              cudaStream_t stream);
// Sets with their own Sobol points (the set table's directions).
cudaError_t launch_k2kf_sets(const nlo_bk_params& p, const double* r, int points, int sets, const double* spline,
                             size_t spline_stride, const int32_t* active, const int32_t* counts,
                             const nlo_bk_box& box, const SetsLayout& L, const SetTable* table, double* out,
                             double* partial, cudaStream_t stream);

// Records a message for nlo_last_error() and returns code.
int set_last_error(int code, const char* message);

// Raise (never lower) a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`; safe when several host threads launch the same kernel with different sizes.
cudaError_t raise_dynamic_smem(const void* func, size_t bytes);
// The BK kernels stage their tables and sample tiles in shared memory and read little through
// L1: ask for the largest shared-memory carveout, once per kernel and device.
cudaError_t prefer_shared_carveout(const void* func);

// Spline tables of `sets` rows: set s reads N.at(s) and writes out + s * spline_doubles(n)
// and its factorisation at factor + s * 2n.
cudaError_t launch_splines(const double* r, const RowsArg& N, int n, int sets, int force_positive, double* factor,
                           int compute_factor, double* out, cudaStream_t stream);
// active parents (index > 0, N <= 0.99999) with index % shards == shard; set s reads N.at(s)
// and writes active + s * n and count + s
cudaError_t launch_active(const RowsArg& N, int n, int sets, int shard, int shards, int32_t* active, int32_t* count,
                          cudaStream_t stream);
cudaError_t launch_sobol(const SobolDirsArg& dirs, uint64_t offset, uint64_t n, int precision, void* out,
                         cudaStream_t stream);
// Amplitude history of the kinematical constraint (bk/derivatives.py:469-487, 712-758):
// rows N[rows][points] at rapidities y[rows], the last row the current amplitude, and
// the per-interval weights of the 6-point natural splines in r (kc_weights_doubles).
struct K1History {
    const double* N = nullptr;
    const double* y = nullptr;
    const double* weights = nullptr;
    int rows = 0;
    bool on = false;
};
constexpr int kKcStride = 14;  // per r interval: start, local interval, 2 x 6 weights
inline size_t kc_weights_doubles(int points) { return (size_t)(points - 1) * kKcStride; }
cudaError_t launch_kc_weights(const double* r, int points, double* weights, cudaStream_t stream);

// K1 of `sets` sets: set s reads spline + s * spline_doubles(points), active + s * points and
// count + s, and writes out + s * points (the constraint history: one set only).
cudaError_t launch_k1(const nlo_bk_params& p, const double* r, int points, const double* spline,
                      const int32_t* active, const int32_t* count, double* out, cudaStream_t stream,
                      const K1History& history = K1History(), int sets = 1);
cudaError_t launch_k2kf(const nlo_bk_params& p, const double* r, int points, const double* spline,
                        const int32_t* active, const int32_t* count, const SobolDirsArg& dirs, uint64_t offset,
                        uint64_t samples, const nlo_bk_box& box, double* out, double* partial, int max_blocks,
                        cudaStream_t stream);
// K2+Kf by Vegas (k2kf_vegas.cu): the per-call buffers, carved from the caller's workspace.
struct BkVegasCall {
    nlo_bk_vegas_options options;
    double* state = nullptr;   // [points][stride], persistent grids
    int stride = 0;
    int blocks_per_job = 1;
    double* partial = nullptr;  // [points][blocks][4 + 4 bins]
    double* reduced = nullptr;  // [points][4 + 4 bins]
    int32_t* counts = nullptr;  // [points][4 bins]
    double* replica_state = nullptr;  // [points][stride], the replicas' fresh grids
    double* replica_acc = nullptr;    // [points][3], the replica refinement's sums
    const SobolDirsArg* replica_dirs = nullptr;  // [options.replicas]
};
size_t bk_vegas_state_doubles(int bins);
int bk_vegas_blocks_per_job(int points);
size_t bk_vegas_scratch_bytes(int points, int bins);
BkVegasCall bk_vegas_carve(void* scratch, int points, const nlo_bk_vegas_options& options, double* state);
// Vegas K2+Kf of the active parents i % shards == shard of N into out[points][3] = [value, 0,
// error^2] (zeros elsewhere).
cudaError_t launch_k2kf_vegas(const nlo_bk_params& p, const double* r, const double* N, int points,
                              const double* spline, int shard, int shards, const SobolDirsArg& dirs,
                              const nlo_bk_box& box, const BkVegasCall& call, double* out, cudaStream_t stream);
// The replica refinement of the parents launch_k2kf_vegas integrated (options.replicas > 0):
// reads their K1 (k1[points]) and the amplitude row N, rewrites out[points][3] of the
// refined parents.
cudaError_t launch_k2kf_vegas_refine(const nlo_bk_params& p, const double* r, const double* N, int points,
                                     const double* spline, const nlo_bk_box& box, const BkVegasCall& call,
                                     const double* k1, double* out, cudaStream_t stream);
// Fixed-order sum of per-CTA partial rows [jobs][blocks][keys] over the CTAs (dis.cu).
cudaError_t vegas_launch_reduce(const double* partial, int keys, int blocks_per_job, int jobs, double* reduced,
                                cudaStream_t stream);

cudaError_t launch_assemble(const double* k1, const double* k2kf, int points, double inv_samples, double* dndy,
                            double* k2kf_total, cudaStream_t stream);
cudaError_t launch_axpy_stage(const double* N, const double* const* k, const double* coef, int nk, int points,
                              double* out, int clamp, uint32_t* status, cudaStream_t stream);
// Several sets: dndy + s * points = k1 + s * points + (k2kf + s * 3 points) * table->inv[s].
cudaError_t launch_assemble_sets(const double* k1, const double* k2kf, int points, int sets, const SetTable* table,
                                 double* dndy, cudaStream_t stream);
// Several sets: out.at(s) = N.at(s) + sum_j coef[j] (k[j] + s * points); status + s when given.
cudaError_t launch_axpy_sets(const RowsArg& N, const double* const* k, const double* coef, int nk, int points,
                             int sets, const RowsArg& out, int clamp, uint32_t* status, cudaStream_t stream);

}  // namespace nlo
