// nlo_bk_k2kf_static: the K2+Kf sums of nlo_bk_k2kf for callers that cannot
// allocate device memory.
//
// Some hosts own the device allocator and do not let this library call
// cudaMalloc: a plugin running inside a framework that has reserved the GPU's
// memory for its own pool, or a serving loop that must not pay cudaMalloc's
// latency and implicit synchronisation on the request path.  Such callers still
// provide the inputs and the output buffer, but cannot provide the scratch that
// nlo_bk_k2kf takes as `workspace`.  This entry point keeps that scratch -- the
// per-CTA partial sums -- in a fixed-size device array defined in this file, so
// it allocates nothing at all.
//
// Limits and sharing:
//  * at most kStaticMaxPoints grid points and kStaticBlocks CTAs; the array
//    holds kStaticBlocks x kStaticMaxPoints x 3 doubles (3.6 MB), and every GPU
//    that loads the library keeps it until the process exits;
//  * the first call on a device looks up the array's device address with that
//    device current (cudaGetSymbolAddress) and caches it; make that first call
//    before any stream capture;
//  * the cached address belongs to the device's context of that first call: after
//    cudaDeviceReset (or anything else that destroys and recreates the primary
//    context) it is stale, so the library must not be used across a device reset;
//  * every call uses the same array, which keeps the last call's contents; each
//    launch writes all the partials it later reads, so nothing needs clearing,
//    but calls that overlap on the GPU (other streams or threads, same device)
//    race on the array and must be serialised by the caller.

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.cuh"
#include "internal.h"

namespace nlo {

namespace {

constexpr int kStaticMaxPoints = 512;
constexpr int kStaticBlocks = 296;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_k2kf_static_scratch[(size_t)kStaticBlocks * kStaticMaxPoints * 3];

std::mutex g_scratch_mutex;
double* g_scratch_address[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per device).
int scratch_on_current_device(double** out)
{
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return set_last_error(NLO_ERR_CUDA, "nlo_bk_k2kf_static: cudaGetDevice failed");
    if (device < 0 || device >= kMaxDevices)
        return set_last_error(NLO_ERR_INVALID, "nlo_bk_k2kf_static: device index beyond 63");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_address[device]) {
        void* address = nullptr;
        e = cudaGetSymbolAddress(&address, g_k2kf_static_scratch);
        if (e != cudaSuccess || !address)
            return set_last_error(NLO_ERR_CUDA, "nlo_bk_k2kf_static: cudaGetSymbolAddress of the scratch array failed");
        g_scratch_address[device] = static_cast<double*>(address);
    }
    *out = g_scratch_address[device];
    return NLO_OK;
}

}  // namespace

}  // namespace nlo

using namespace nlo;

extern "C" int nlo_bk_k2kf_static(const nlo_bk_params* params, const double* r, int32_t points,
                                  const double* spline, const int32_t* active, const int32_t* count,
                                  const nlo_sobol_dirs* dirs, int64_t offset, int64_t samples,
                                  const nlo_bk_box* box, double* out, void* stream)
{
    if (!r || !spline || !active || !count || !out || !box)
        return set_last_error(NLO_ERR_INVALID, "nlo_bk_k2kf_static: NULL argument");
    // the same parameter and direction-number checks as nlo_bk_k2kf, so both K2+Kf entry
    // points accept and reject the same inputs
    std::string why;
    if (!check_params(params, why)) return set_last_error(NLO_ERR_INVALID, ("nlo_bk_k2kf_static: " + why).c_str());
    if (!check_dirs(dirs, 4, why)) return set_last_error(NLO_ERR_INVALID, ("nlo_bk_k2kf_static: " + why).c_str());
    if (points < 3 || points > kStaticMaxPoints)
        return set_last_error(NLO_ERR_INVALID,
                              "nlo_bk_k2kf_static: points must be 3..512 (the fixed scratch array's limit); "
                              "use nlo_bk_k2kf with a workspace for larger grids");
    if (offset < 0 || samples < 0 || offset + samples > (int64_t(1) << 30))
        return set_last_error(NLO_ERR_INVALID, "nlo_bk_k2kf_static: Sobol index range exceeds 2^30");
    double* scratch = nullptr;
    const int rc = scratch_on_current_device(&scratch);
    if (rc != NLO_OK) return rc;
    const cudaError_t e = launch_k2kf(*params, r, points, spline, active, count, to_arg(dirs), (uint64_t)offset,
                                      (uint64_t)samples, *box, out, scratch, kStaticBlocks, (cudaStream_t)stream);
    if (e != cudaSuccess) return set_last_error(NLO_ERR_CUDA, cudaGetErrorString(e));
    return NLO_OK;
}
