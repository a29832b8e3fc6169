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
//  * every call uses the same array, which keeps the last call's contents; each
//    launch writes all the partials it later reads, so nothing needs clearing,
//    but calls that overlap on the GPU (other streams or threads, same device)
//    race on the array and must be serialised by the caller.

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

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
    if (!params || !dirs || !box || !r || !spline || !active || !count || !out)
        return set_last_error(NLO_ERR_INVALID, "nlo_bk_k2kf_static: NULL argument");
    if (!(params->nc > 0) || !(params->nf == 0.0 || params->nf == 3.0 || params->nf == 5.0) ||
        !(params->lambda_qcd > 0) || !(params->c2 > 0) || !(params->ksub > 0) ||
        (params->rc_nlo != NLO_RC_NLO_SMALLEST && params->rc_nlo != NLO_RC_NLO_PARENT) ||
        (params->precision != NLO_PRECISION_MIXED && params->precision != NLO_PRECISION_FP64))
        return set_last_error(NLO_ERR_INVALID, "nlo_bk_k2kf_static: unsupported physics parameters");
    if (dirs->dims < 4 || dirs->dims > 8)
        return set_last_error(NLO_ERR_INVALID, "nlo_bk_k2kf_static: Sobol dimension count out of range");
    for (int j = 0; j < dirs->dims; ++j) {
        if (dirs->shift[j] >= (1u << 30))
            return set_last_error(NLO_ERR_INVALID, "nlo_bk_k2kf_static: Sobol shift exceeds 30 bits");
        for (int k = 0; k < 30; ++k)
            if (dirs->state[j][k] >= (1u << 30))
                return set_last_error(NLO_ERR_INVALID, "nlo_bk_k2kf_static: Sobol direction number exceeds 30 bits");
    }
    if (points < 3 || points > kStaticMaxPoints)
        return set_last_error(NLO_ERR_INVALID,
                              "nlo_bk_k2kf_static: points must be 3..512 (the fixed scratch array's limit); "
                              "use nlo_bk_k2kf with a workspace for larger grids");
    if (offset < 0 || samples < 0 || offset + samples > (int64_t(1) << 30))
        return set_last_error(NLO_ERR_INVALID, "nlo_bk_k2kf_static: Sobol index range exceeds 2^30");
    double* scratch = nullptr;
    const int rc = scratch_on_current_device(&scratch);
    if (rc != NLO_OK) return rc;
    SobolDirsArg arg;
    std::memset(&arg, 0, sizeof(arg));
    arg.dims = dirs->dims;
    std::memcpy(arg.state, dirs->state, sizeof(arg.state));
    std::memcpy(arg.shift, dirs->shift, sizeof(arg.shift));
    const cudaError_t e = launch_k2kf(*params, r, points, spline, active, count, arg, (uint64_t)offset,
                                      (uint64_t)samples, *box, out, scratch, kStaticBlocks, (cudaStream_t)stream);
    if (e != cudaSuccess) return set_last_error(NLO_ERR_CUDA, cudaGetErrorString(e));
    return NLO_OK;
}
