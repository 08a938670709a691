// pb_noalloc.cu -- the WET pass for callers that cannot allocate device
// memory.
//
// pb_wet needs a work buffer of n_beams x V floats for the unsmoothed WET,
// and its caller provides it.  Some callers cannot: code embedded in a host
// framework that owns the whole device pool (an XLA/JAX custom call, whose
// allocator has preallocated most of the GPU and which hands the call only
// its input and output buffers), or a planning-system plug-in that is given
// device buffers and may not create its own.  pb_wet_noalloc serves them:
// its work space is a file-scope device array of this library, so the call
// allocates nothing.
//
// The array holds PB_NOALLOC_MAX_WET_FLOATS floats (32 MiB).  Every GPU on
// which the library's device code is loaded holds it until the process
// exits.  Requests with n_beams x V above that size are rejected.  All calls
// share the one array: calls that overlap on the GPU (different streams,
// different host threads on the same device) race on it and must be
// serialised by the caller.  Each call overwrites every element it later
// reads (the ray trace writes the raw WET of every voxel of every beam
// before the smoothing reads any), so nothing needs clearing between calls.
//
// Host code cannot use the array's name as a device address.  The entry
// point asks the runtime for the array's address in the current context
// (cudaGetSymbolAddress, with the device current) on its first call in that
// context, and keeps it for that context: one set-up per device, repeated
// only if the device's context is re-created (after cudaDeviceReset, say).
#include <cuda.h>

#include <mutex>

#include "pb_internal.h"

namespace pb {

static __device__ __align__(256) float g_noalloc_raw_wet[PB_NOALLOC_MAX_WET_FLOATS];

constexpr int kNoallocDevices = 64;
static std::mutex g_noalloc_mu;
static CUcontext g_noalloc_ctx[kNoallocDevices];
static float *g_noalloc_addr[kNoallocDevices];

using CtxGetCurrent = CUresult (*)(CUcontext *);

// The driver's cuCtxGetCurrent, found through the runtime (the library does
// not link libcuda itself).
static CtxGetCurrent ctx_get_current()
{
    static CtxGetCurrent fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault,
                                             &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<CtxGetCurrent>(p);
    }();
    return fn;
}

// Device address of the work array in the current device's context.
static PbStatus noalloc_scratch(float **out)
{
    int dev = -1;
    PbStatus s = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (s != PB_OK) return s;
    if (dev < 0 || dev >= kNoallocDevices)
        return set_error(PB_ERR_UNSUPPORTED, "device ordinal %d is beyond %d", dev,
                         kNoallocDevices);
    // cudaFree(0) makes the device's primary context current (no allocation)
    s = check_cuda(cudaFree(nullptr), "cudaFree(0) (context set-up)");
    if (s != PB_OK) return s;
    CtxGetCurrent get = ctx_get_current();
    CUcontext ctx = nullptr;
    if (!get || get(&ctx) != CUDA_SUCCESS || !ctx)
        return set_error(PB_ERR_CUDA, "pb_wet_noalloc: no current CUDA context");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev] || g_noalloc_ctx[dev] != ctx) {
        void *p = nullptr;
        s = check_cuda(cudaGetSymbolAddress(&p, g_noalloc_raw_wet),
                       "cudaGetSymbolAddress(work array)");
        if (s != PB_OK) return s;
        g_noalloc_addr[dev] = static_cast<float *>(p);
        g_noalloc_ctx[dev] = ctx;
    }
    *out = g_noalloc_addr[dev];
    return PB_OK;
}

}  // namespace pb

using namespace pb;

extern "C" PbStatus pb_wet_noalloc(const float *rlsp_dev, PbTexture tex, const PbGrid *grid,
                                   const PbBeamGeom *beams, int n_beams, float *wet_dev,
                                   int *status_dev, void *stream)
{
    // the same inputs as pb_wet accepts, less its work buffer
    PbStatus s = check_wet_args(rlsp_dev, tex, grid, beams, n_beams, wet_dev);
    if (s != PB_OK) return s;
    const double need = (double)n_beams * grid->nx * grid->ny * grid->nz;
    if (need > (double)PB_NOALLOC_MAX_WET_FLOATS)
        return set_error(PB_ERR_INVALID,
                         "pb_wet_noalloc: n_beams x voxels = %.0f exceeds its fixed work "
                         "space of %u floats; use pb_wet with a caller-provided buffer",
                         need, (unsigned)PB_NOALLOC_MAX_WET_FLOATS);
    float *raw = nullptr;
    s = noalloc_scratch(&raw);
    if (s != PB_OK) return s;
    return launch_wet(rlsp_dev, texture_object(tex), texture_cells(tex), *grid, beams, n_beams,
                      raw, wet_dev, status_dev, static_cast<cudaStream_t>(stream));
}
