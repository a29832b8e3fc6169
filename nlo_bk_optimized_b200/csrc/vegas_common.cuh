// Device pieces of the Vegas integrator shared by the DIS terms (dis.cu) and the BK K2+Kf
// integral (k2kf_vegas.cu): the grid re-binning of _adapt_vegas_edges
// (numerics/integration.py:804-866) and the inverse-variance combination of the iteration
// estimates with the convergence test (:510-582).  Both run in one CTA per integral, in a
// fixed order, so results are bit-reproducible.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nlo {
namespace vegas {

// Slots after the edges [D][bins+1] of a per-integral state.
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

// New edges of every dimension from the |w| histogram and the bin counts: importance =
// hist / max(count, 1), three-point smoothing (two at the ends), + DBL_EPSILON, equal-mass
// re-binning of the cumulative importance against the old edges; the end edges stay 0 and 1.
// Called by all threads of the CTA; smooth [D*bins], cum [D*(bins+1)] and next [D*(bins+1)]
// are shared-memory scratch.  edges is read and then overwritten.
__device__ inline void rebin(double* edges, const double* hist, const int32_t* counts, int D, int bins,
                             double* smooth, double* cum, double* next)
{
    for (int k = threadIdx.x; k < D * bins; k += blockDim.x) {
        const int d = k / bins, b = k % bins;
        auto imp = [&](int q) {
            const int n = counts[d * bins + q];
            return hist[d * bins + q] / (double)(n > 1 ? n : 1);
        };
        double v;
        if (b == 0)
            v = (imp(0) + imp(1)) / 2.0;
        else if (b == bins - 1)
            v = (imp(bins - 2) + imp(bins - 1)) / 2.0;
        else
            v = (imp(b - 1) + imp(b) + imp(b + 1)) / 3.0;
        smooth[k] = v + 2.220446049250313e-16;
    }
    __syncthreads();
    if (threadIdx.x < D) {
        const int d = threadIdx.x;
        double* cd = cum + d * (bins + 1);
        cd[0] = 0.0;
        for (int b = 0; b < bins; ++b) cd[b + 1] = cd[b] + smooth[d * bins + b];
        const double* e = edges + d * (bins + 1);
        double* out = next + d * (bins + 1);
        const double total = cd[bins];
        const double step = total / bins;
        int idx = 0;
        for (int k = 0; k <= bins; ++k) {
            // torch.linspace(0, total, bins + 1); the targets increase, so the
            // searchsorted(right) - 1 index only moves forward
            const double target = k < (bins + 1) / 2 ? step * k : total - step * (bins - k);
            while (idx < bins && cd[idx + 1] <= target) ++idx;
            const int i = idx > bins - 1 ? bins - 1 : idx;
            const double frac = (target - cd[i]) / smooth[d * bins + i];
            out[k] = e[i] + frac * (e[i + 1] - e[i]);
        }
        out[0] = 0.0;
        out[bins] = 1.0;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < D * (bins + 1); k += blockDim.x) edges[k] = next[k];
}

// One reported iteration of `samples` weights with sum s and sum of squares s2: its
// estimate and variance join the inverse-variance-weighted combination in the scalar slots
// sc; value, error and the convergence flag (after min_iterations, error <= max(epsabs,
// epsrel |value|)) are updated.  Returns the iteration's weight 1/variance.
__device__ inline double combine(double* sc, double s, double s2, double samples, int min_iterations, double epsrel,
                                 double epsabs)
{
    const double n = samples;
    const double est = s / n;
    double var = (s2 - s * s / n);
    var = var > 0.0 ? var : 0.0;
    var = var / (n - 1.0) / n;
    var = var > 2.2250738585072014e-308 ? var : 2.2250738585072014e-308;
    sc[kStSumWeightedEst] += est / var;
    sc[kStSumWeights] += 1.0 / var;
    sc[kStIterations] += 1.0;
    sc[kStLastEstimate] = est;
    sc[kStLastVariance] = var;
    const double value = sc[kStSumWeightedEst] / sc[kStSumWeights];
    const double error = ::sqrt(1.0 / sc[kStSumWeights]);
    sc[kStValue] = value;
    sc[kStError] = error;
    const double tol = epsabs > epsrel * ::fabs(value) ? epsabs : epsrel * ::fabs(value);
    if (sc[kStIterations] >= (double)min_iterations && error <= tol) sc[kStConverged] = 1.0;
    return 1.0 / var;
}

}  // namespace vegas
}  // namespace nlo
