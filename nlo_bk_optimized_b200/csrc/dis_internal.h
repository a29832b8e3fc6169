// Internal launch interfaces of the DIS kernels (dis.cu) used by the C ABI (dis_capi.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "internal.h"

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

// Per-integral Vegas state: edges[D][bins+1] followed by these scalar slots.
enum StateSlot {
    kStSumWeightedEst = 0,  // sum of estimate / variance over reported iterations
    kStSumWeights = 1,      // sum of 1 / variance
    kStValue = 2,
    kStError = 3,
    kStEvals = 4,
    kStIterations = 5,
    kStConverged = 6,
    kStLastEstimate = 7,
    kStLastVariance = 8,
    kStSlots = 16,
};

struct VegasLaunch {
    const void* args;            // device DisArgs<T>[jobs]
    const SobolDirsArg* dirs;    // device [jobs]
    const InnerRule* rule;       // host copy (passed by value)
    double* state;               // device [jobs][state_stride]
    int state_stride;
    int jobs, bins, blocks_per_job;
    uint64_t offset, samples;
    double* partial;             // device [jobs][blocks][2 + D*bins]
    int32_t* counts;             // device [jobs][blocks][D*bins]
    int warmup, min_iterations;
    double epsrel, epsabs;
};

}  // namespace dis

cudaError_t dis_launch_table_prepare(const double* r, const double* y, const double* N, int nr, int ny, double y0,
                                     double* table, cudaStream_t stream);
cudaError_t dis_launch_table_initialize(double* table, int nr, int ny, double Y, cudaStream_t stream);
cudaError_t dis_launch_points(int precision, int term, const void* args, const dis::InnerRule& rule, const double* x,
                              int64_t n, double* out, cudaStream_t stream);
cudaError_t dis_launch_amplitude(int precision, const void* args, const double* r, const double* Y, int64_t n,
                                 double* out, cudaStream_t stream);
cudaError_t dis_launch_gl(int precision, int term, const void* args, int jobs, const dis::InnerRule& rule,
                          const dis::GLRules& gl, double* out, cudaStream_t stream);
cudaError_t dis_launch_vegas_init(double* state, int state_stride, int D, int bins, int jobs, int keep_edges,
                                  cudaStream_t stream);
cudaError_t dis_launch_vegas_round(int precision, int term, const dis::VegasLaunch& L, cudaStream_t stream);

// Gauss-Legendre nodes and weights on [-1, 1], ascending (capi.cu)
void gauss_legendre_rule(int n, double* x, double* w);

}  // namespace nlo
