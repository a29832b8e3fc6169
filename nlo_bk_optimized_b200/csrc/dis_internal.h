// Internal launch interfaces of the DIS kernels (dis.cu) used by the C ABI (dis_capi.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "internal.h"
#include "vegas_common.cuh"

namespace nlo {
namespace dis {

struct InnerRule;

constexpr int kVegasThreads = 256;
constexpr int kMaxBins = 256;

// Tensor Gauss-Legendre rules on [0, 1] (fine and half order).
struct GLRules {
    int n_fine, n_coarse;
    double x_fine[64], w_fine[64];
    double x_coarse[32], w_coarse[32];
};

// Per-integral Vegas state: edges[D][bins+1] followed by the scalar slots of
// vegas_common.cuh (kSt*).
using vegas::StateSlot;
using vegas::kStSumWeightedEst;
using vegas::kStSumWeights;
using vegas::kStValue;
using vegas::kStError;
using vegas::kStEvals;
using vegas::kStIterations;
using vegas::kStConverged;
using vegas::kStLastEstimate;
using vegas::kStLastVariance;
using vegas::kStSlots;

struct VegasLaunch {
    const void* args;            // device DisArgs<T>[jobs]
    const SobolDirsArg* dirs;    // device [jobs]
    const InnerRule* rule;       // host copy (passed by value)
    double* state;               // device [jobs][state_stride]
    int state_stride;
    int jobs, bins, blocks_per_job;
    uint64_t offset, samples;
    double* partial;             // device [jobs][blocks][2 + D*bins]
    double* reduced;             // device [jobs][2 + D*bins]
    int32_t* counts;             // device [jobs][D*bins], integer sums over the CTAs
    int warmup, min_iterations;
    double epsrel, epsabs;
};

}  // namespace dis

cudaError_t dis_launch_table_prepare(const double* r, const double* y, const double* N, int nr, int ny, double y0,
                                     int interp, double* table, cudaStream_t stream);
cudaError_t dis_launch_table_initialize(double* table, int nr, int ny, double Y, cudaStream_t stream);
cudaError_t dis_launch_points(int precision, int term, const void* args, const dis::InnerRule& rule, const double* x,
                              int64_t n, double* out, cudaStream_t stream);
cudaError_t dis_launch_amplitude(int precision, const void* args, const double* r, const double* Y, int64_t n,
                                 double* out, cudaStream_t stream);
cudaError_t dis_launch_gl(int precision, int term, const void* args, int jobs, const dis::InnerRule& rule,
                          const dis::GLRules& gl, double* out, cudaStream_t stream);
cudaError_t dis_launch_vegas_init(double* state, int state_stride, int D, int bins, int jobs, int keep_edges,
                                  int32_t* counts, cudaStream_t stream);
cudaError_t dis_launch_vegas_round(int precision, int term, const dis::VegasLaunch& L, cudaStream_t stream);
// Reduce per-CTA partials [jobs][blocks][2 + D*bins] and run the grid adaptation and
// estimate update of one Vegas round (warmup = adaptation only).
cudaError_t dis_launch_reduce_finalize(int D, int bins, int jobs, int blocks_per_job, const double* partial,
                                       double* reduced, int32_t* counts, double* state, int state_stride,
                                       uint64_t samples, int warmup, int min_iterations, double epsrel, double epsabs,
                                       cudaStream_t stream);

// Fixed-Sobol qqbar-g integration (dis_fixed.cu).  The workspace starts with the
// Sobol directions of the training rounds and replicates (SobolDirsArg each).
bool dis_fixed_check(const nlo_fixed_sobol_options* o, std::string& why);
size_t dis_fixed_workspace_bytes(const nlo_fixed_sobol_options& o);
int dis_run_fixed(int precision, const void* args, const dis::InnerRule& rule, const nlo_fixed_sobol_options& o,
                  void* workspace, double* grid_state, double* estimates, cudaStream_t s);

// Gauss-Legendre nodes and weights on [-1, 1], ascending (capi.cu)
void gauss_legendre_rule(int n, double* x, double* w);

}  // namespace nlo
