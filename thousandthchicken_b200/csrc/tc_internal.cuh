// tc_internal.cuh -- shared declarations of the CUDA side of libtc_j2k.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "tc_j2k.h"

// Device error word bits (set by kernels, read by tc_ctx_synchronize).
#define TC_DERR_DESC 0x1u     // a code-block descriptor was out of range
#define TC_DERR_POOL 0x2u     // a codeword ran past the segment pool
#define TC_DERR_STYLE 0x4u    // a styled code-block reached a style-0 launch, or its segment table is bad
#define TC_DERR_OUT 0x8u      // a code-block's place ran past the output (block skipped, nothing written)
#define TC_DERR_TIMEOUT 0x10u // a bounded device wait (an mbarrier of a TMA copy) gave up

namespace tc {

// One-time setup per device shared by every context (kernel attributes,
// occupancy): fn runs once per device under a lock, and its results are
// published to the other threads by the release store of the flag.
inline std::mutex &device_setup_mutex()
{
    static std::mutex m;
    return m;
}
using DeviceFlags = std::atomic<bool>[64];
template <typename F>
cudaError_t once_per_device(DeviceFlags &done, int device, F &&fn)
{
    std::atomic<bool> &d = done[device & 63];
    if (d.load(std::memory_order_acquire)) return cudaSuccess;
    std::lock_guard<std::mutex> lock(device_setup_mutex());
    if (d.load(std::memory_order_relaxed)) return cudaSuccess;
    const cudaError_t e = fn();
    if (e == cudaSuccess) d.store(true, std::memory_order_release);
    return e;
}
// cudaFuncSetAttribute(kernel, max dynamic shared memory) once per device.
template <typename K>
cudaError_t set_smem_once(DeviceFlags &done, int device, K kernel, size_t smem)
{
    return once_per_device(done, device, [&] {
        return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
}

// Code-block style bits that change decoding (PTERM only constrains the
// encoder's terminations).
constexpr int kStyleDecodeBits = TC_CBLK_STYLE_BYPASS | TC_CBLK_STYLE_RESET | TC_CBLK_STYLE_TERMALL |
                                 TC_CBLK_STYLE_VSC | TC_CBLK_STYLE_SEGSYM;

// Sample range of an output of `bits` bits (TC_SIGNED set: signed samples,
// two's complement, no DC level shift; ISO G.1.2 shifts unsigned ones only).
struct OutRange {
    int dc, lo, hi;
};
__host__ __device__ inline OutRange out_range(int bits)
{
    const int b = bits & 0xFF;
    if (bits & TC_SIGNED) return OutRange{0, -(1 << (b - 1)), (1 << (b - 1)) - 1};
    return OutRange{1 << (b - 1), 0, (1 << b) - 1};
}

// Grow-only device buffer owned by a context.
struct DevBuf {
    void *ptr = nullptr;
    size_t size = 0;
    cudaStream_t stream = nullptr;  // set by ensure_on: stream-ordered allocation
    bool ordered = false;
    cudaError_t ensure(size_t bytes);
    // Grows through the stream-ordered allocator (memory pool `pool`) on
    // `s`: the old block is freed after the work already queued on `s`, and
    // no call waits for the rest of the device (cudaFree would).
    cudaError_t ensure_on(size_t bytes, cudaStream_t s, cudaMemPool_t pool);
    void release();
};

// Pinned host staging buffer (grow-only).
struct PinBuf {
    void *ptr = nullptr;
    size_t size = 0;
    // Outgrown blocks.  cudaFreeHost waits for the whole device, which in a
    // serving loop means another batch in flight, so they are only freed
    // with the buffer itself.
    std::vector<void *> retired;
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= size && ptr) return cudaSuccess;
        // doubling: a serving loop's batches vary, and every regrowth re-pins
        const size_t want = bytes < 4096 ? 4096 : (bytes < 2 * size ? 2 * size : bytes);
        if (ptr) retired.push_back(ptr);
        ptr = nullptr;
        size = 0;
        cudaError_t e = cudaHostAlloc(&ptr, want, cudaHostAllocDefault);
        if (e == cudaSuccess) size = want;
        else ptr = nullptr;
        return e;
    }
    void release()
    {
        if (ptr) cudaFreeHost(ptr);
        for (void *p : retired) cudaFreeHost(p);
        retired.clear();
        ptr = nullptr;
        size = 0;
    }
};

}  // namespace tc

struct tc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    uint32_t *d_words = nullptr;  // [0] error word, [1..6] Tier-1 work counters
    tc::DevBuf scratch;           // DWT intermediate levels
    tc::DevBuf tmp_pool, tmp_desc, tmp_order, tmp_coef, tmp_out;
    tc::PinBuf stage_pool, stage_desc, stage_order;  // pinned staging of tc_decode_j2k
    // tc_encode_j2k_gpu's buffers (samples, colour planes, coefficients,
    // Tier-1 descriptors, codewords, results, offsets, packed codewords);
    // grow-only, so repeated encodes allocate nothing after the first
    tc::DevBuf enc[8];
    tc::PinBuf enc_host;          // the packed codewords read back
    // reverse-DWT job table of tc_decode_j2k's tiled images
    tc::DevBuf tmp_jobs;
    tc::PinBuf stage_jobs;
    cudaEvent_t jobs_uploaded = nullptr;
    uint64_t launches = 0;
    int t1_group = 32;            // lanes per code-block in the Tier-1 kernel (8, 16 or 32)
    int dwt_variant = TC_DWT_TMA; // staging of the fused last reverse 9/7 level (TC_DWT_*)
    // side streams for concurrent Tier-1 class launches (created on first use)
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    // stream that plan graphs are captured on (the caller's stream may be the
    // legacy default stream, which cannot be captured)
    cudaStream_t capture = nullptr;
    // device memory pool of the plans' buffers; it keeps freed memory mapped
    // (release threshold: unlimited) so that regrowth does not map again
    cudaMemPool_t pool = nullptr;
};

namespace tc {

// The context's memory pool (created on first use).
cudaError_t ctx_mem_pool(tc_ctx *ctx, cudaMemPool_t *out);
// Creates the context's side streams, capture stream and fork/join events
// if needed.
cudaError_t ensure_side_streams(tc_ctx *ctx);
// Records a message on the context and returns the status.
int fail(tc_ctx *ctx, int status, const std::string &msg);
// Maps a CUDA error to TC_E_DEVICE with its message (TC_OK on cudaSuccess).
int cuda_status(tc_ctx *ctx, cudaError_t e, const char *what);

// ---- kernels' host launchers (each returns a cudaError_t of the launch) ----

// One persistent launch over n blocks whose coded bit-planes are at most
// max_bitplanes (selects the magnitude storage width: 8, 16 or 32 bits).
cudaError_t launch_t1_decode(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order,
                             int n, const uint8_t *d_pool, uint64_t pool_len, void *d_out,
                             uint64_t out_elems, int out_mode, float recon_r, int max_bitplanes);
// Persistent launches over an order array partitioned into blocks of at
// most 8, 16 and 31 coded bit-planes (n8 + n16 + n32 entries), then blocks
// with a code-block style in the same three widths (nstyled[0..2], or none).
cudaError_t launch_t1_classes(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order,
                              int ndesc, int n8, int n16, int n32, const uint8_t *d_pool,
                              uint64_t pool_len, void *d_out, uint64_t out_elems, int out_mode,
                              float recon_r, const int *nstyled = nullptr);
// Host: order longest-first within each class (<= 8, <= 16, <= 31 coded
// bit-planes, then styled blocks of <= 8, <= 16, <= 31); class sizes out.
void t1_class_order(const tc_cblk_desc *h_desc, int n, uint32_t *h_order, int counts[6]);
cudaError_t launch_dequant_raw(tc_ctx *ctx, const tc_cblk_desc *d_desc, int n,
                               const uint32_t *d_raw, void *d_out, uint64_t elems, float recon_r);
cudaError_t launch_t1_encode(tc_ctx *ctx, const tc_t1_enc_desc *d_desc, int n, const void *d_in, uint8_t *d_out,
                             uint32_t cap, tc_t1_enc_result *d_res);
// Packs n codewords (block k: res[k].len bytes at src + k * cap) to dst + off[k].
cudaError_t launch_gather_codewords(tc_ctx *ctx, const uint8_t *src, uint32_t cap, const tc_t1_enc_result *res,
                                    const uint64_t *off, int n, uint8_t *dst);

// One 2-D DWT level over up to 4 components of equal size.
struct LevelIO {
    const void *ll[4];     // reverse: LL input; forward: spatial input
    const void *coef[4];   // reverse: Mallat plane holding HL/LH/HH of the level
    void *out[4];          // reverse: samples of the level; forward: LL output
    void *bands[4];        // forward: Mallat plane receiving HL/LH/HH
    int ll_pitch, coef_pitch, out_pitch, bands_pitch;
    int w, h;              // size of the level's full-resolution region
    int ncomp;
};

// wavelet: 0 = 5/3 int32, 1 = 9/7 float.  rounding: TC_ROUND_*.
cudaError_t launch_idwt_level(tc_ctx *ctx, const LevelIO &io, int wavelet, int rounding);

// A reverse level of one plane (plane levels) or one image (last level with
// colour) inside a batched launch; tile0 is the index of its first tile among
// the launch's tiles, tiles_x its tiles per row (see rev_tile_shape).
struct RevJob {
    LevelIO io;
    int tiles_x;
    int tile0;
};
void rev_tile_shape(int wavelet, int *tx, int *ty);
// One launch over the jobs d_jobs[0..njobs) (device memory, tile0 ascending,
// ntiles tiles in all), all of one kind: plane levels when color < 0 (each
// job one component), else last levels with colour of ncomp components
// writing out_type samples of `bits` bits.
cudaError_t launch_idwt_batch(tc_ctx *ctx, const RevJob *d_jobs, int njobs, int ntiles, int wavelet, int rounding,
                              int color, int ncomp, int out_type, int bits);
cudaError_t launch_fdwt_level(tc_ctx *ctx, const LevelIO &io, int wavelet, int rounding);

// Last reverse 9/7 level of a three-component image with the inverse ICT
// fused in, packed fp32x2 lifting (dwt_rev97.cu).  rev97_handles says
// whether a last level runs there (ICT, 3 components, 8- or 16-bit out).
bool rev97_handles(int color, int ncomp, int out_type);
cudaError_t launch_rev97_level(tc_ctx *ctx, const LevelIO &io, int out_type, int bits);
cudaError_t launch_rev97_batch(tc_ctx *ctx, const RevJob *d_jobs, int njobs, int ntiles, int out_type, int bits);
// The same last level with its subband tiles staged by TMA (dwt_tma.cu), for
// levels whose band width, pitches and addresses suit 2-D tensor copies
// (rev97_tma_handles).
bool rev97_tma_handles(const LevelIO &io, int out_type);
cudaError_t launch_rev97_tma(tc_ctx *ctx, const LevelIO &io, int out_type, int bits);

// Last reverse level fused with the inverse colour transform, DC shift,
// rounding and clamping; writes out_type samples (TC_U8/TC_U16/TC_INT32).
// color: TC_COLOR_DC / TC_COLOR_RCT / TC_COLOR_ICT.  levels == 0 means the
// input is already spatial (no lifting).
cudaError_t launch_idwt_last_color(tc_ctx *ctx, const LevelIO &io, int wavelet, int color,
                                   int out_type, int bits, bool lift);

// Standalone colour kernels.
cudaError_t launch_color_inverse(tc_ctx *ctx, int kind, int ncomp, void *const *in, int in_type,
                                 int in_pitch, void *const *out, int out_type, int out_pitch,
                                 int w, int h, int bits);
cudaError_t launch_color_forward(tc_ctx *ctx, int kind, int ncomp, const void *const *in,
                                 int in_type, int in_pitch, void *const *out, int out_type,
                                 int out_pitch, int w, int h, int bits);

inline int num_sms(int device)
{
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
    return n;
}

}  // namespace tc
