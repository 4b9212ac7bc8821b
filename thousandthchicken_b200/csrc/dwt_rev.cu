// dwt_rev.cu -- reverse DWT levels (5/3 int32, 9/7 fp32) for sm_100a.
//
// One CTA reconstructs a 128-column output tile of one level (56 rows for
// 9/7, 60 for 5/3): it loads the 64-row extended tile (a halo of H = 4 or 2
// samples on every side) straight from the level's four subbands into shared
// memory, with whole-sample symmetric extension (ISO F.3.7; the reference's
// single reflection, dwt_io.cl:7-38, is defect D14), then
//   * horizontal lifting: each thread lifts one 32-sample segment of one row
//     (plus its halo) entirely in registers, fully unrolled, reading and
//     writing it with 16-byte shared-memory accesses;
//   * vertical lifting: two threads per column each lift an overlapping half
//     (36 rows for 9/7, 34 for 5/3) in registers and store it (coalesced
//     across the warp);
// so every lifting step is register arithmetic with constant indices and the
// CTA synchronises only between phases.  The row stride in shared memory is
// a multiple of four words with an odd quotient, so threads walking
// different rows hit different banks.
//
// COLOR >= 0 fuses the inverse RCT/ICT, DC shift, rounding and clamp into the
// store of the last level (the reference's tcr_kernel / tci_kernel /
// idc_level_shift_kernel, Preprocessor.cpp:44-180), writing 8/16-bit samples:
// the last component's column is combined in registers with the other two,
// parked in shared memory.  The ISO 2D_SR order is kept: rows first, then
// columns (DWTReverse53/97, dwt_r53.cl / dwt_r97.cl).
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "dwt_common.cuh"
#include "tc_internal.cuh"

namespace tc {
namespace {

using namespace dwt;

constexpr int kThreads = 256;

template <int WAVELET>
struct RevGeo {
    static constexpr int H = WAVELET ? 4 : 2;     // halo
    static constexpr int NR = 64;                 // extended rows per tile
    static constexpr int TY = NR - 2 * H;         // output rows per tile
    static constexpr int TX = 128;                // output columns per tile
    static constexpr int NC = TX + 2 * H;         // extended columns
    // row stride: a multiple of 4 words (16-byte rows for 128-bit access)
    // with S/4 odd, so 8 threads reading 16 bytes each from 8 consecutive
    // rows cover all 32 banks once
    static constexpr int S = (NC % 8 == 4) ? NC : NC + 4;
    static constexpr int SEG = 32;                // outputs per row segment
    static constexpr int SEGN = SEG + 2 * H;      // inputs per row segment
};

// In-place 1-D reverse lifting of an interleaved signal held in registers
// (v[0] at an even position; even = low-pass).  Only samples at least H away
// from both ends are exact.
template <typename T, int WAVELET, int RND, int N>
__device__ __forceinline__ void lift_reverse(T (&v)[N])
{
    if constexpr (WAVELET == 0) {
#pragma unroll
        for (int k = 2; k <= N - 2; k += 2) v[k] -= div4r<RND>(v[k - 1] + v[k + 1] + 2);
#pragma unroll
        for (int k = 1; k <= N - 3; k += 2) v[k] += div2r<RND>(v[k - 1] + v[k + 1]);
    } else {
        // scaling-free form: the K / 1/K factors of ISO F.3.8.2 steps 1-2
        // are folded into the constants (E/K and O*K are lifted), and the
        // caller applies the remaining per-parity factor once per output
#pragma unroll
        for (int k = 2; k <= N - 2; k += 2) v[k] = fmaf(-kSfD, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
        for (int k = 1; k <= N - 3; k += 2) v[k] = fmaf(-kSfG, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
        for (int k = 2; k <= N - 2; k += 2) v[k] = fmaf(-kSfB, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
        for (int k = 1; k <= N - 3; k += 2) v[k] = fmaf(-kSfA, v[k - 1] + v[k + 1], v[k]);
    }
}

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <typename OT>
__device__ __forceinline__ OT clamp_out(int v, const OutRange &R)
{
    return (OT)(v < R.lo ? R.lo : (v > R.hi ? R.hi : v));
}

template <typename T>
__device__ __forceinline__ int to_int(T v)
{
    if constexpr (std::is_same<T, float>::value) return __float2int_rn(v);
    else return (int)v;
}

// 16-byte vector of four T (T is int32_t or float).
template <typename T>
using Vec4 = typename std::conditional<std::is_same<T, float>::value, float4, int4>::type;

// Phase 1 of a tile: issues the asynchronous copies of tile (bx, by) of
// level `io`, NT components from cbase, into `tiles` (the caller waits).
template <typename T, int WAVELET, int NT>
__device__ __forceinline__ void rev_stage(const LevelIO &io, int bx, int by, int cbase, T *tiles)
{
    using G = RevGeo<WAVELET>;
    constexpr int H = G::H, NR = G::NR, TY = G::TY, TX = G::TX, NC = G::NC, S = G::S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int x0 = bx * TX, y0 = by * TY;
    const int w = io.w, h = io.h, wl = (w + 1) >> 1, hl = (h + 1) >> 1;

    // 1. load the extended tiles from the four subbands (Mallat layout) with
    //    4-byte asynchronous copies, so a thread has its whole share of the
    //    tile in flight at once.  x0 - H is even, so the parity of a column
    //    is the parity of the lane: inside the plane a lane's sources in a
    //    row are one strided run of the low or the high band.
    const bool interior = x0 >= H && x0 + TX + H <= w && y0 >= H && y0 + NR - H <= h;
#pragma unroll
    for (int cc = 0; cc < NT; cc++) {
        T *t = tiles + cc * NR * S;
        const T *ll = static_cast<const T *>(io.ll[cbase + cc]);
        const T *coef = static_cast<const T *>(io.coef[cbase + cc]);
        if (interior) {
            // y0 - H is even and a warp's rows step by 8: a warp copies rows
            // of one parity only, so each lane's source is one band row
            // advancing by 4 rows of its plane per step
            constexpr int RSTEP = kThreads / 32;
            static_assert(RSTEP % 2 == 0, "a warp's rows share a parity");
            const int xs = ((x0 - H) >> 1) + (lane >> 1);
            const int y = y0 - H + warp, yb = y >> 1;
            const bool from_ll = !(y & 1) && !(lane & 1);
            const size_t pitch = from_ll ? (size_t)io.ll_pitch : (size_t)io.coef_pitch;
            const T *src = (y & 1) ? coef + (size_t)(hl + yb) * io.coef_pitch + ((lane & 1) ? wl : 0)
                                   : ((lane & 1) ? coef + (size_t)yb * io.coef_pitch + wl
                                                 : ll + (size_t)yb * io.ll_pitch);
            src += xs;
            const size_t step = pitch * (RSTEP / 2);
            T *dst = t + warp * S + lane;
#pragma unroll 2
            for (int r = warp; r < NR; r += RSTEP, src += step, dst += RSTEP * S) {
#pragma unroll
                for (int j = 0; j < NC / 32; j++) cp_async4(dst + 32 * j, src + 16 * j);
                if (lane < NC % 32) cp_async4(dst + 32 * (NC / 32), src + 16 * (NC / 32));
            }
        } else {
            for (int r = warp; r < NR; r += kThreads / 32) {
                const int my = mirror(y0 - H + r, h), yb = my >> 1;
                const T *lrow = (my & 1) ? coef + (size_t)(hl + yb) * io.coef_pitch : ll + (size_t)yb * io.ll_pitch;
                const T *hrow = coef + (size_t)((my & 1) ? hl + yb : yb) * io.coef_pitch + wl;
#pragma unroll
                for (int e = lane; e < NC; e += 32) {
                    const int mx = mirror(x0 - H + e, w);
                    cp_async4(t + r * S + e, ((mx & 1) ? hrow : lrow) + (mx >> 1));
                }
            }
        }
    }
}

// Phases 2-3 of a staged tile: lifting and the store.
template <typename T, int WAVELET, int RND, int NCOMP, int COLOR, typename OT>
__device__ __forceinline__ void rev_compute(const LevelIO &io, int bits, int bx, int by, int cbase, T *tiles)
{
    using G = RevGeo<WAVELET>;
    constexpr int H = G::H, NR = G::NR, TY = G::TY, TX = G::TX, S = G::S;
    constexpr bool PLANE = COLOR < 0;
    constexpr int NT = PLANE ? 1 : NCOMP;
    const int tid = threadIdx.x;
    const int x0 = bx * TX, y0 = by * TY;
    const int w = io.w, h = io.h;

    // 2. horizontal lifting, one row segment per thread (64 rows x 4
    //    segments of 32 outputs); segments are read and written with 16-byte
    //    (8-byte for the 2-sample halo of 5/3) shared-memory accesses
    static_assert(NR * (TX / G::SEG) == kThreads, "one row segment per thread");
    if (w > 1) {
        const int seg = tid / NR, r = tid % NR;  // a warp walks 32 consecutive rows
#pragma unroll
        for (int cc = 0; cc < NT; cc++) {
            T *row = tiles + cc * NR * S + r * S + seg * G::SEG;
            T v[G::SEGN];
#pragma unroll
            for (int k = 0; k < G::SEGN; k += 4) {
                const Vec4<T> q = *reinterpret_cast<const Vec4<T> *>(row + k);
                v[k] = q.x;
                v[k + 1] = q.y;
                v[k + 2] = q.z;
                v[k + 3] = q.w;
            }
            __syncthreads();  // neighbouring segments overlap: all reads before any write
            lift_reverse<T, WAVELET, RND, G::SEGN>(v);
            if constexpr (H % 4 == 0) {
#pragma unroll
                for (int k = H; k < H + G::SEG; k += 4) {
                    Vec4<T> q;
                    q.x = v[k];
                    q.y = v[k + 1];
                    q.z = v[k + 2];
                    q.w = v[k + 3];
                    *reinterpret_cast<Vec4<T> *>(row + k) = q;
                }
            } else {
                using V2 = typename std::conditional<std::is_same<T, float>::value, float2, int2>::type;
#pragma unroll
                for (int k = H; k < H + G::SEG; k += 2) {
                    V2 q;
                    q.x = v[k];
                    q.y = v[k + 1];
                    *reinterpret_cast<V2 *>(row + k) = q;
                }
            }
        }
        __syncthreads();
    }

    // 3. vertical lifting, two threads per column, and the store.  The top
    //    thread lifts rows [0, 32 + H) and keeps output rows [0, 32 - H); the
    //    bottom one lifts rows [32 - H, 64) and keeps [32 - H, TY).  With a
    //    colour transform the first two components are parked in their own
    //    tiles, in rows that only the parking thread reads: the top thread at
    //    rows [0, 32 - H), the bottom one at [NR - (32 - H), NR).  The third
    //    component's column is then combined with them from registers.
    constexpr int VN = 32 + H, OUTR = 32 - H;
    const int col = tid % TX, half = tid / TX, x = x0 + col;
    const int vbase = half ? 32 - H : 0;             // first tile row lifted
    const int obase = half ? OUTR : 0;               // first output row kept
    const int pbase = half ? NR - OUTR : 0;          // first parking row
    const bool full_rows = y0 + obase + OUTR <= h;
    const OutRange R = out_range(PLANE ? 8 : bits);
    const int dc = PLANE ? 0 : R.dc;
#pragma unroll
    for (int cc = 0; cc < NT; cc++) {
        T *t = tiles + cc * NR * S;
        T v[VN];
#pragma unroll
        for (int k = 0; k < VN; k++) v[k] = t[(vbase + k) * S + H + col];
        if (h > 1) lift_reverse<T, WAVELET, RND, VN>(v);
        if constexpr (WAVELET == 1) {
            // x0 and the first kept row are even: parities are col & 1, r & 1
            const float fe = sf_factor(0, col & 1, w > 1, h > 1), fo = sf_factor(1, col & 1, w > 1, h > 1);
#pragma unroll
            for (int r = 0; r < OUTR; r++) v[H + r] *= (r & 1) ? fo : fe;
        }
        if (x >= w) continue;
        const int y = y0 + obase;
        if constexpr (PLANE) {
            T *out = static_cast<T *>(io.out[cbase]) + (size_t)y * io.out_pitch + x;
            const size_t pitch = (size_t)io.out_pitch;
            if (full_rows) {
#pragma unroll
                for (int r = 0; r < OUTR; r++, out += pitch) *out = v[H + r];
            } else {
#pragma unroll
                for (int r = 0; r < OUTR; r++, out += pitch)
                    if (y + r < h) *out = v[H + r];
            }
        } else if (COLOR == TC_COLOR_DC || cc >= 3) {
            OT *out = static_cast<OT *>(io.out[cc]) + (size_t)y * io.out_pitch + x;
#pragma unroll
            for (int r = 0; r < OUTR; r++)
                if (full_rows || y + r < h) out[(size_t)r * io.out_pitch] = clamp_out<OT>(to_int(v[H + r]) + dc, R);
        } else if (cc < 2) {
#pragma unroll
            for (int r = 0; r < OUTR; r++) t[(pbase + r) * S + H + col] = v[H + r];
        } else {
            const T *t0 = tiles + (pbase * S + H + col), *t1 = tiles + (NR * S + pbase * S + H + col);
            const size_t o = (size_t)y * io.out_pitch + x;
            OT *o0 = static_cast<OT *>(io.out[0]) + o, *o1 = static_cast<OT *>(io.out[1]) + o,
               *o2 = static_cast<OT *>(io.out[2]) + o;
#pragma unroll
            for (int r = 0; r < OUTR; r++) {
                if (!(full_rows || y + r < h)) continue;
                int c0, c1, c2;
                if constexpr (COLOR == TC_COLOR_RCT) {
                    const int Y = (int)t0[r * S], U = (int)t1[r * S], V = (int)v[H + r];
                    const int Gc = Y - ((U + V) >> 2);
                    c0 = V + Gc;
                    c1 = Gc;
                    c2 = U + Gc;
                } else {
                    const float Y = (float)t0[r * S], Cb = (float)t1[r * S], Cr = (float)v[H + r];
                    c0 = __float2int_rn(fmaf(1.402f, Cr, Y));
                    c1 = __float2int_rn(Y - 0.34413f * Cb - 0.71414f * Cr);
                    c2 = __float2int_rn(fmaf(1.772f, Cb, Y));
                }
                const size_t ro = (size_t)r * io.out_pitch;
                o0[ro] = clamp_out<OT>(c0 + dc, R);
                o1[ro] = clamp_out<OT>(c1 + dc, R);
                o2[ro] = clamp_out<OT>(c2 + dc, R);
            }
        }
    }
}

// The CTA's work: tile (bx, by) of level `io`, components from cbase.
template <typename T, int WAVELET, int RND, int NCOMP, int COLOR, typename OT>
__device__ __forceinline__ void rev_tile(const LevelIO &io, int bits, int bx, int by, int cbase)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *tiles = reinterpret_cast<T *>(smem_raw);
    rev_stage<T, WAVELET, COLOR < 0 ? 1 : NCOMP>(io, bx, by, cbase, tiles);
    cp_async_wait_all();
    __syncthreads();
    rev_compute<T, WAVELET, RND, NCOMP, COLOR, OT>(io, bits, bx, by, cbase, tiles);
}

// One level of one image: tiles (blockIdx.x, blockIdx.y), one component per
// blockIdx.z for plane levels.
template <typename T, int WAVELET, int RND, int NCOMP, int COLOR, typename OT>
__global__ void __launch_bounds__(kThreads) idwt_rev_kernel(LevelIO io, int bits)
{
    pdl_allow_next();
    pdl_wait_prev();
    rev_tile<T, WAVELET, RND, NCOMP, COLOR, OT>(io, bits, blockIdx.x, blockIdx.y, COLOR < 0 ? blockIdx.z : 0);
}

// One level of many images (or planes) of mixed sizes in one launch: the
// jobs' tiles are numbered consecutively (job j owns tiles
// [jobs[j].tile0, jobs[j+1].tile0)), and each CTA finds its job by binary
// search.
template <typename T, int WAVELET, int RND, int NCOMP, int COLOR, typename OT>
__global__ void __launch_bounds__(kThreads) idwt_rev_batch_kernel(const RevJob *__restrict__ jobs, int njobs,
                                                                  int bits)
{
    pdl_allow_next();
    const int b = blockIdx.x;
    int lo = 0, hi = njobs - 1;   // the job table is written by the host before any level runs
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].tile0 <= b) lo = mid;
        else hi = mid - 1;
    }
    const RevJob &J = jobs[lo];
    const int t = b - J.tile0;
    pdl_wait_prev();
    rev_tile<T, WAVELET, RND, NCOMP, COLOR, OT>(J.io, bits, t % J.tiles_x, t / J.tiles_x, 0);
}

template <typename T, int WAVELET, int NCOMP, int COLOR>
constexpr size_t rev_smem()
{
    return (size_t)(COLOR < 0 ? 1 : NCOMP) * RevGeo<WAVELET>::NR * RevGeo<WAVELET>::S * sizeof(T);
}

// A launch of one level: a single image (batch == nullptr, io given) or the
// jobs of a batch (njobs jobs, ntiles tiles in all).
struct RevLaunch {
    const LevelIO *io = nullptr;
    const RevJob *jobs = nullptr;
    int njobs = 0, ntiles = 0;
};

template <typename T, int WAVELET, int RND, int NCOMP, int COLOR, typename OT>
cudaError_t run_rev(tc_ctx *ctx, const RevLaunch &L, int bits)
{
    using G = RevGeo<WAVELET>;
    constexpr size_t smem = rev_smem<T, WAVELET, NCOMP, COLOR>();
    cudaError_t e;
    if (L.io) {
        static DeviceFlags attr;
        if ((e = set_smem_once(attr, ctx->device, idwt_rev_kernel<T, WAVELET, RND, NCOMP, COLOR, OT>, smem)) !=
            cudaSuccess)
            return e;
        const LevelIO &io = *L.io;
        dim3 grid((io.w + G::TX - 1) / G::TX, (io.h + G::TY - 1) / G::TY, COLOR < 0 ? io.ncomp : 1);
        if ((e = launch_pdl(idwt_rev_kernel<T, WAVELET, RND, NCOMP, COLOR, OT>, grid, dim3(kThreads), smem,
                            ctx->stream, io, bits)) != cudaSuccess)
            return e;
    } else {
        if (L.njobs <= 0 || L.ntiles <= 0) return cudaSuccess;
        static DeviceFlags attr;
        if ((e = set_smem_once(attr, ctx->device, idwt_rev_batch_kernel<T, WAVELET, RND, NCOMP, COLOR, OT>, smem)) !=
            cudaSuccess)
            return e;
        if ((e = launch_pdl(idwt_rev_batch_kernel<T, WAVELET, RND, NCOMP, COLOR, OT>, dim3(L.ntiles),
                            dim3(kThreads), smem, ctx->stream, L.jobs, L.njobs, bits)) != cudaSuccess)
            return e;
    }
    ctx->launches++;
    return cudaGetLastError();
}

template <typename T, int WAVELET, int RND, int COLOR>
cudaError_t run_last(tc_ctx *ctx, const RevLaunch &L, int ncomp, int out_type, int bits)
{
#define TC_LAST(NC_)                                                                        \
    (out_type == TC_U8    ? run_rev<T, WAVELET, RND, NC_, COLOR, uint8_t>(ctx, L, bits)  \
     : out_type == TC_U16 ? run_rev<T, WAVELET, RND, NC_, COLOR, uint16_t>(ctx, L, bits) \
                          : run_rev<T, WAVELET, RND, NC_, COLOR, int32_t>(ctx, L, bits))
    if (COLOR != TC_COLOR_DC) return ncomp == 4 ? TC_LAST(4) : TC_LAST(3);
    switch (ncomp) {
    case 1: return TC_LAST(1);
    case 2: return TC_LAST(2);
    case 3: return TC_LAST(3);
    default: return TC_LAST(4);
    }
#undef TC_LAST
}

cudaError_t plane_level(tc_ctx *ctx, const RevLaunch &L, int wavelet, int rounding)
{
    if (wavelet) return run_rev<float, 1, 0, 1, -1, float>(ctx, L, 0);
    if (rounding == TC_ROUND_TRUNC) return run_rev<int32_t, 0, TC_ROUND_TRUNC, 1, -1, int32_t>(ctx, L, 0);
    return run_rev<int32_t, 0, TC_ROUND_FLOOR, 1, -1, int32_t>(ctx, L, 0);
}

cudaError_t last_level(tc_ctx *ctx, const RevLaunch &L, int ncomp, int wavelet, int color, int out_type, int bits)
{
    if (color != TC_COLOR_DC && ncomp < 3) color = TC_COLOR_DC;
    if (wavelet) {
        if (color == TC_COLOR_ICT || color == TC_COLOR_RCT)
            return run_last<float, 1, 0, TC_COLOR_ICT>(ctx, L, ncomp, out_type, bits);
        return run_last<float, 1, 0, TC_COLOR_DC>(ctx, L, ncomp, out_type, bits);
    }
    if (color == TC_COLOR_RCT || color == TC_COLOR_ICT)
        return run_last<int32_t, 0, TC_ROUND_FLOOR, TC_COLOR_RCT>(ctx, L, ncomp, out_type, bits);
    return run_last<int32_t, 0, TC_ROUND_FLOOR, TC_COLOR_DC>(ctx, L, ncomp, out_type, bits);
}

}  // namespace

cudaError_t launch_idwt_level(tc_ctx *ctx, const LevelIO &io, int wavelet, int rounding)
{
    if (io.w <= 0 || io.h <= 0) return cudaSuccess;
    RevLaunch L;
    L.io = &io;
    return plane_level(ctx, L, wavelet, rounding);
}

cudaError_t launch_idwt_last_color(tc_ctx *ctx, const LevelIO &io, int wavelet, int color, int out_type, int bits,
                                   bool)
{
    if (io.w <= 0 || io.h <= 0) return cudaSuccess;
    if (color != TC_COLOR_DC && io.ncomp < 3) color = TC_COLOR_DC;
    if (wavelet && rev97_handles(color, io.ncomp, out_type)) {
        if (ctx->dwt_variant == TC_DWT_TMA && rev97_tma_handles(io, out_type))
            return launch_rev97_tma(ctx, io, out_type, bits);
        return launch_rev97_level(ctx, io, out_type, bits);
    }
    RevLaunch L;
    L.io = &io;
    return last_level(ctx, L, io.ncomp, wavelet, color, out_type, bits);
}

void rev_tile_shape(int wavelet, int *tx, int *ty)
{
    *tx = wavelet ? RevGeo<1>::TX : RevGeo<0>::TX;
    *ty = wavelet ? RevGeo<1>::TY : RevGeo<0>::TY;
}

cudaError_t launch_idwt_batch(tc_ctx *ctx, const RevJob *d_jobs, int njobs, int ntiles, int wavelet, int rounding,
                              int color, int ncomp, int out_type, int bits)
{
    if (color >= 0 && color != TC_COLOR_DC && ncomp < 3) color = TC_COLOR_DC;
    if (wavelet && rev97_handles(color, ncomp, out_type))
        return launch_rev97_batch(ctx, d_jobs, njobs, ntiles, out_type, bits);
    RevLaunch L;
    L.jobs = d_jobs;
    L.njobs = njobs;
    L.ntiles = ntiles;
    if (color < 0) return plane_level(ctx, L, wavelet, rounding);
    return last_level(ctx, L, ncomp, wavelet, color, out_type, bits);
}

}  // namespace tc
