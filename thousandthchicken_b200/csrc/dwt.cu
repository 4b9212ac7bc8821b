// dwt.cu -- forward 5/3 (int32) and 9/7 (fp32) lifting DWT levels for
// sm_100a (the encoder's and the tc_dwt_forward* entry points; the reverse
// levels are in dwt_rev.cu).
//
// Replaces the reference's forward kernels (dwt_f53.cl, dwt_f97.cl over
// dwt_transform_buffer.cl / dwt_io.cl).  One 256-thread CTA transforms a tile
// of 120 output columns by 56 (9/7) or 60 (5/3) output rows of one level:
//   * it stages the extended tile (halo of H = 4 or 2 samples on every side)
//     in shared memory with 4-byte asynchronous copies, whole-sample
//     symmetric extension at the image edges (ISO F.3.7; the reference's
//     single reflection, dwt_io.cl:7-38, is defect D14);
//   * vertical lifting first (ISO 2D_SD: columns, then rows): two threads
//     per column each lift an overlapping half of it in registers;
//   * horizontal lifting: one thread per 30-output row segment, in
//     registers, whose low- and high-pass results go back to shared memory
//     de-interleaved;
//   * the store writes each row's low and high halves to the level's LL and
//     HL (even rows) or LH and HH (odd rows) bands, coalesced.
// 5/3 uses floor (ISO) or truncating (reference, defect D13) rounding; 9/7
// uses fp32 with the scaling factors applied as floats (defects D10-D12
// fixed).  The lifting steps and their order follow ISO F.4.8.
#include <cuda_runtime.h>

#include <type_traits>

#include "dwt_common.cuh"
#include "tc_internal.cuh"

namespace tc {
namespace {

using namespace dwt;

constexpr int kThreads = 256;

template <int WAVELET>
struct FwdGeo {
    static constexpr int H = WAVELET ? 4 : 2;     // halo
    static constexpr int NR = 64;                 // extended rows per tile
    static constexpr int TY = NR - 2 * H;         // output rows per tile
    static constexpr int TX = 120;                // output columns per tile (even)
    static constexpr int NC = TX + 2 * H;         // extended columns
    static constexpr int S = (NC % 8 == 4) ? NC : NC + 4;  // row stride, S/4 odd
    static constexpr int SEG = 30;                // outputs per row segment (even)
    static constexpr int SEGN = SEG + 2 * H;      // inputs per row segment
    static constexpr int VN = 32 + H;             // rows lifted by one thread of a column pair
    static constexpr int OUTV = 32 - H;           // rows it keeps
};

// In-place 1-D forward lifting of a signal held in registers (v[0] at an
// even position).  Only samples at least H away from both ends are exact.
template <typename T, int WAVELET, int RND, int N>
__device__ __forceinline__ void lift_forward(T (&v)[N])
{
    if constexpr (WAVELET == 0) {
#pragma unroll
        for (int k = 1; k <= N - 2; k += 2) v[k] -= div2r<RND>(v[k - 1] + v[k + 1]);
#pragma unroll
        for (int k = 2; k <= N - 2; k += 2) v[k] += div4r<RND>(v[k - 1] + v[k + 1] + 2);
    } else {
#pragma unroll
        for (int k = 1; k <= N - 2; k += 2) v[k] = fmaf(kA, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
        for (int k = 2; k <= N - 2; k += 2) v[k] = fmaf(kB, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
        for (int k = 1; k <= N - 2; k += 2) v[k] = fmaf(kG, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
        for (int k = 2; k <= N - 2; k += 2) v[k] = fmaf(kD, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
        for (int k = 0; k + 1 < N; k += 2) {
            v[k] *= kInvK;
            v[k + 1] *= kK;
        }
    }
}

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Forward level, one component per blockIdx.z: io.ll[c] is the spatial input
// (pitch ll_pitch), io.out[c] receives LL (out_pitch), io.bands[c] the Mallat
// plane holding HL/LH/HH (bands_pitch).
template <typename T, int WAVELET, int RND>
__global__ void __launch_bounds__(kThreads) fdwt_level_kernel(LevelIO io)
{
    using G = FwdGeo<WAVELET>;
    constexpr int H = G::H, NR = G::NR, TY = G::TY, TX = G::TX, NC = G::NC, S = G::S;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *t = reinterpret_cast<T *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int c = blockIdx.z;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int w = io.w, h = io.h;
    const T *in = static_cast<const T *>(io.ll[c]);

    // 1. stage the extended tile
    const bool interior = x0 >= H && x0 - H + NC <= w && y0 >= H && y0 - H + NR <= h;
    for (int r = warp; r < NR; r += kThreads / 32) {
        const int y = interior ? y0 - H + r : mirror(y0 - H + r, h);
        const T *row = in + (size_t)y * io.ll_pitch;
        for (int e = lane; e < NC; e += 32) {
            const int x = interior ? x0 - H + e : mirror(x0 - H + e, w);
            cp_async4(t + r * S + e, row + x);
        }
    }
    cp_async_wait_all();
    __syncthreads();

    // 2. vertical lifting: column pairs of threads, rows [0, VN) and
    //    [NR - VN, NR); the results go back in place once all have read
    {
        const int col = tid % 128, half = tid / 128;
        const int vbase = half ? NR - G::VN : 0;
        T v[G::VN];
        if (col < NC) {
#pragma unroll
            for (int k = 0; k < G::VN; k++) v[k] = t[(vbase + k) * S + col];
        }
        __syncthreads();
        if (col < NC) {
            if (h > 1) lift_forward<T, WAVELET, RND, G::VN>(v);
#pragma unroll
            for (int k = 0; k < G::OUTV; k++) t[(vbase + H + k) * S + col] = v[H + k];
        }
        __syncthreads();
    }

    // 3. horizontal lifting of the TY output rows, one 30-output segment per
    //    thread; low outputs go to row words [0, TX/2), high to [64, 64 + TX/2)
    {
        constexpr int NSEG = TX / G::SEG;
        const bool active = tid < TY * NSEG;
        const int seg = tid / TY, r = H + tid % TY;  // a warp walks consecutive rows
        T v[G::SEGN];
        if (active) {
#pragma unroll
            for (int k = 0; k < G::SEGN; k++) v[k] = t[r * S + seg * G::SEG + k];
        }
        __syncthreads();  // segments overlap, and the outputs overwrite the inputs
        if (active) {
            if (w > 1) lift_forward<T, WAVELET, RND, G::SEGN>(v);
#pragma unroll
            for (int i = 0; i < G::SEG / 2; i++) {
                t[r * S + seg * (G::SEG / 2) + i] = v[H + 2 * i];
                t[r * S + 64 + seg * (G::SEG / 2) + i] = v[H + 2 * i + 1];
            }
        }
        __syncthreads();
    }

    // 4. store: row by row, the low half to LL / LH, the high half to HL / HH;
    //    a thread keeps one of the 120 output slots of a row (60 low, 60 high)
    //    and walks every other row
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    constexpr int HALF = TX / 2;
    const int j = tid % 128, r0 = tid / 128;
    if (j < TX) {
        const bool hi = j >= HALF;
        const int i = hi ? j - HALF : j;
        const int x = x0 + 2 * i + (hi ? 1 : 0);
        if (x < w) {
            const int xb = (x0 >> 1) + i;
            T *ll = static_cast<T *>(io.out[c]) + xb;
            T *bands = static_cast<T *>(io.bands[c]) + xb + (hi ? wl : 0);
            const T *src = t + (hi ? 64 : 0) + i;
            for (int r = r0; r < TY && y0 + r < h; r += 2) {
                const int y = y0 + r, yb = y >> 1;
                const T val = src[(H + r) * S];
                if (y & 1) bands[(size_t)(hl + yb) * io.bands_pitch] = val;
                else if (hi) bands[(size_t)yb * io.bands_pitch] = val;
                else ll[(size_t)yb * io.out_pitch] = val;
            }
        }
    }
}

template <typename T, int WAVELET, int RND>
cudaError_t run_fdwt(tc_ctx *ctx, const LevelIO &io)
{
    using G = FwdGeo<WAVELET>;
    constexpr size_t smem = (size_t)G::NR * G::S * sizeof(T);
    static DeviceFlags attr;
    if (cudaError_t e = set_smem_once(attr, ctx->device, fdwt_level_kernel<T, WAVELET, RND>, smem)) return e;
    dim3 grid((io.w + G::TX - 1) / G::TX, (io.h + G::TY - 1) / G::TY, io.ncomp);
    fdwt_level_kernel<T, WAVELET, RND><<<grid, kThreads, smem, ctx->stream>>>(io);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_fdwt_level(tc_ctx *ctx, const LevelIO &io, int wavelet, int rounding)
{
    if (io.w <= 0 || io.h <= 0) return cudaSuccess;
    if (wavelet) return run_fdwt<float, 1, 0>(ctx, io);
    if (rounding == TC_ROUND_TRUNC) return run_fdwt<int32_t, 0, TC_ROUND_TRUNC>(ctx, io);
    return run_fdwt<int32_t, 0, TC_ROUND_FLOOR>(ctx, io);
}

}  // namespace tc
