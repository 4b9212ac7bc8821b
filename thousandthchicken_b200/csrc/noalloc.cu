// noalloc.cu -- reverse 9/7 DWT for callers that must not allocate device
// memory.
//
// Some callers cannot call cudaMalloc.  Examples: code running inside a CUDA
// stream capture that must not allocate, hosts whose memory manager owns
// every device allocation, and real-time paths where an allocation (and the
// device synchronisation cudaFree implies) would stall the pipeline.  This
// entry point gives them the multi-level reverse 9/7 transform without any
// allocation.  The intermediate LL plane that tc_dwt_reverse97 keeps in a
// grow-only buffer of its context lives here in one file-scope device array
// of fixed size.  The caller passes the input and output planes; nothing
// else is touched.
//
// Contract:
//  * The array holds TC_DWT97_STATIC_SCRATCH_ELEMS floats (16 MiB).  Every
//    GPU that loads this library keeps it until the process exits.
//    Transforms whose first-level low band, ceil(w/2) * ceil(h/2), is larger
//    are rejected with TC_E_ARG before any work is issued.
//  * The first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it for the
//    life of the process.  Make that first call outside any stream capture.
//    The cached address does not survive cudaDeviceReset on that device
//    (the module, and the array with it, may be reloaded elsewhere): do not
//    call this entry point on a device after resetting it.
//  * All calls share the one array.  Two calls whose work overlaps on the
//    GPU (different streams, or different host threads) race on it; order
//    them on one stream or serialise them.
//  * The array keeps whatever the last call left in it.  Nothing needs to
//    start at zero: every intermediate sample is written by a level before
//    the next level reads it.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "j2k_host.h"
#include "tc_internal.cuh"

namespace {

__device__ __align__(256) float g_dwt97_scratch[TC_DWT97_STATIC_SCRATCH_ELEMS];

std::mutex g_setup_mu;
float *g_scratch_ptr[64] = {};

// Device address of g_dwt97_scratch on the current device (resolved once).
cudaError_t static_scratch(int device, float **out)
{
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_dwt97_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[device] = static_cast<float *>(p);
    }
    *out = g_scratch_ptr[device];
    return cudaSuccess;
}

}  // namespace

extern "C" int tc_dwt_reverse97_static(const float *d_in, int in_pitch, float *d_out, int out_pitch, int w, int h,
                                       int levels, void *cuda_stream)
{
    if (!d_in || !d_out || d_in == d_out || w <= 0 || h <= 0 || in_pitch < w || out_pitch < w || levels < 0 ||
        levels > 32)
        return TC_E_ARG;
    std::vector<int> ws, hs;
    tc::level_sizes(w, h, levels, ws, hs);
    if (levels >= 2 && (size_t)ws[1] * (size_t)hs[1] > (size_t)TC_DWT97_STATIC_SCRATCH_ELEMS)
        return TC_E_ARG;  // the intermediate plane does not fit the static array
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    // The array's address is resolved on every device's first call, whatever
    // the level count, so that a caller's first call does the lookup outside
    // any capture even when it has nothing to transform.
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return TC_E_DEVICE;
    float *scratch = nullptr;
    if (static_scratch(device, &scratch) != cudaSuccess) return TC_E_DEVICE;
    if (levels == 0) {
        const cudaError_t e = cudaMemcpy2DAsync(d_out, (size_t)out_pitch * 4, d_in, (size_t)in_pitch * 4,
                                                (size_t)w * 4, h, cudaMemcpyDeviceToDevice, stream);
        return e == cudaSuccess ? TC_OK : TC_E_DEVICE;
    }

    // A context on the stack: the launchers only read its device and
    // stream and count launches; it owns no memory.
    tc_ctx local;
    local.device = device;
    local.stream = stream;
    // Levels alternate between the output plane (odd levels) and the static
    // array (even levels), so no level reads the plane it writes; the
    // deepest level reads its LL band from the input.
    const float *src = d_in;
    int src_pitch = in_pitch;
    for (int l = levels; l >= 1; l--) {
        tc::LevelIO io{};
        io.w = ws[l - 1];
        io.h = hs[l - 1];
        io.ncomp = 1;
        io.ll[0] = src;
        io.ll_pitch = src_pitch;
        io.coef[0] = d_in;
        io.coef_pitch = in_pitch;
        if (l & 1) {
            io.out[0] = d_out;
            io.out_pitch = out_pitch;
        } else {
            io.out[0] = scratch;
            io.out_pitch = ws[1];
        }
        if (tc::launch_idwt_level(&local, io, 1, TC_ROUND_FLOOR) != cudaSuccess) return TC_E_DEVICE;
        src = static_cast<const float *>(io.out[0]);
        src_pitch = io.out_pitch;
    }
    return TC_OK;
}
