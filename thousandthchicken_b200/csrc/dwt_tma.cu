// dwt_tma.cu -- the last reverse 9/7 level of a three-component image with
// the inverse ICT fused in, its subband tiles staged by TMA.
//
// The kernel of dwt_rev97.cu stages its 64 x 136 extended tile with one
// 4-byte asynchronous copy per sample, because the Mallat subbands
// interleave every other column; those copies fill the shared-memory
// instruction queue.  Here one thread issues twelve 2-D tensor copies
// (cp.async.bulk.tensor, no multicast) per CTA: for each component the
// tile's part of the four subbands (LL, HL, LH, HH), 32 band rows x 72 band
// columns each, completed on one mbarrier.  The lifting works on the band
// arrays as they land:
//   * extended row r (plane row y0 - 4 + r) is band row r / 2 of the low
//     (r even: LL and HL) or the high (r odd: LH and HH) rows; extended
//     column e is band column e / 2 + 2 of the low (e even) or the high
//     (e odd) array;
//   * the horizontal pass reads a row segment's low and high samples from
//     the two arrays, interleaves them in registers, lifts, and writes the
//     results back de-interleaved in place;
//   * the vertical pass lifts each column from the alternating row arrays,
//     Y and Cb paired as fp32x2 (FADD2/FFMA2), Cr alone, then the inverse
//     ICT, DC shift, rounding and saturation, as in dwt_rev97.cu.
// Tiles that touch the plane's border: the copies read zeros (or other
// bands' samples, always finite) outside the band; the columns and then the
// rows within 4 of the border are rebuilt by whole-sample symmetric
// extension (ISO F.3.7) from the staged tile.  The mbarrier wait is bounded:
// a copy that never lands sets the context's error word and the CTA returns.
//
// Applies when the level is at least 16 x 16, its low band width, the row
// pitches of both planes and their addresses are multiples of 16 bytes (TMA
// box coordinates and strides); other levels keep the cp.async kernel.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <type_traits>

#include "dwt_common.cuh"
#include "tc_internal.cuh"

namespace tc {
namespace {

using namespace dwt;

constexpr int kThreads = 256;
constexpr int H = 4, NR = 64, TY = NR - 2 * H, TX = 128;
constexpr int BW = 72, BR = 32;        // band box: 72 band columns x 32 band rows
constexpr int BOX = BW * BR;           // floats per box
constexpr int COMPF = 4 * BOX;         // floats per component: LL, HL, LH, HH
constexpr uint32_t kBoxBytes = BOX * 4;
constexpr uint32_t kTileBytes = 12 * kBoxBytes;
constexpr size_t kSmem = (size_t)3 * COMPF * 4 + 16;   // + the mbarrier
constexpr int SEG = 32, SEGN = SEG + 2 * H;
constexpr int VN = 32 + H, OUTR = 32 - H;
static_assert(kBoxBytes % 128 == 0, "every box starts 128-byte aligned");

struct alignas(64) IctMaps {
    CUtensorMap ll[3];     // the level's low band (LL input) of each component: wl x hl
    CUtensorMap coef[3];   // the level's region of each component's Mallat plane: w x h
};

// Array of extended row r and column parity p within a component's boxes:
// 0 LL (even rows, low columns), 1 HL, 2 LH (odd rows, low columns), 3 HH.
__device__ __forceinline__ float *band_row(float *comp, int r, int p)
{
    return comp + ((r & 1) * 2 + p) * BOX + (r >> 1) * BW;
}
// Cell of extended row r, extended column e.
__device__ __forceinline__ float &cell(float *comp, int r, int e) { return band_row(comp, r, e & 1)[(e >> 1) + 2]; }

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <int N>
__device__ __forceinline__ void lift2(float2 (&v)[N])
{
    const float2 c1 = f2(-kSfD, -kSfD), c2 = f2(-kSfG, -kSfG), c3 = f2(-kSfB, -kSfB), c4 = f2(-kSfA, -kSfA);
#pragma unroll
    for (int k = 2; k <= N - 2; k += 2) v[k] = fma2(c1, add2(v[k - 1], v[k + 1]), v[k]);
#pragma unroll
    for (int k = 1; k <= N - 3; k += 2) v[k] = fma2(c2, add2(v[k - 1], v[k + 1]), v[k]);
#pragma unroll
    for (int k = 2; k <= N - 2; k += 2) v[k] = fma2(c3, add2(v[k - 1], v[k + 1]), v[k]);
#pragma unroll
    for (int k = 1; k <= N - 3; k += 2) v[k] = fma2(c4, add2(v[k - 1], v[k + 1]), v[k]);
}

template <int N>
__device__ __forceinline__ void lift1(float (&v)[N])
{
#pragma unroll
    for (int k = 2; k <= N - 2; k += 2) v[k] = fmaf(-kSfD, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
    for (int k = 1; k <= N - 3; k += 2) v[k] = fmaf(-kSfG, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
    for (int k = 2; k <= N - 2; k += 2) v[k] = fmaf(-kSfB, v[k - 1] + v[k + 1], v[k]);
#pragma unroll
    for (int k = 1; k <= N - 3; k += 2) v[k] = fmaf(-kSfA, v[k - 1] + v[k + 1], v[k]);
}

template <typename OT>
__device__ __forceinline__ OT to_out(float v, const OutRange &R, bool sgn)
{
    int r;
    if constexpr (std::is_same<OT, uint8_t>::value) {
        if (sgn) asm("cvt.rni.sat.s8.f32 %0, %1;" : "=r"(r) : "f"(v));
        else asm("cvt.rni.sat.u8.f32 %0, %1;" : "=r"(r) : "f"(v));
        if (R.hi < 127 || (!sgn && R.hi < 255)) r = min(max(r, R.lo), R.hi);
    } else {
        if (sgn) asm("cvt.rni.sat.s16.f32 %0, %1;" : "=r"(r) : "f"(v));
        else asm("cvt.rni.sat.u16.f32 %0, %1;" : "=r"(r) : "f"(v));
        if (R.hi < 32767 || (!sgn && R.hi < 65535)) r = min(max(r, R.lo), R.hi);
    }
    return (OT)r;
}

// ---- TMA and mbarrier (PTX) ----------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// A bounded wait for phase `phase` of the mbarrier: false after about a
// second without completion.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase)
{
    for (int i = 0; i < (1 << 20); i++) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// One 2-D box of `map` at element coordinates (x, y) into shared memory at
// dst, completing `bar`'s transaction count.  x * 4 bytes is a multiple of 16.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// ---- the tile ------------------------------------------------------------------

struct TileArgs {
    int w, h, out_pitch, bits;
    void *out[3];
};

// Horizontal pass of one row segment: thread (r, s) lifts outputs
// [32 s, 32 s + 32) of extended row r, of the Y/Cb pair (PAIR) or of Cr.
template <bool PAIR>
__device__ __forceinline__ void hpass(float *c0, float *c1, int r, int s)
{
    using V = typename std::conditional<PAIR, float2, float>::type;
    const int j0 = 16 * s + 2;   // band column of the segment's first input
    V v[SEGN];
    {
        // 16-byte loads from band column j0 - 2 (a multiple of 4): 24 cells
        // per array, of which cells 2 .. 21 are the segment's inputs
        const float *al = band_row(c0, r, 0) + j0 - 2, *ah = band_row(c0, r, 1) + j0 - 2;
        const float *bl = band_row(c1, r, 0) + j0 - 2, *bh = band_row(c1, r, 1) + j0 - 2;
        float L0[24], H0[24], L1[PAIR ? 24 : 1], H1[PAIR ? 24 : 1];
#pragma unroll
        for (int k = 0; k < 24; k += 4) {
            const float4 a = *reinterpret_cast<const float4 *>(al + k), b = *reinterpret_cast<const float4 *>(ah + k);
            L0[k] = a.x, L0[k + 1] = a.y, L0[k + 2] = a.z, L0[k + 3] = a.w;
            H0[k] = b.x, H0[k + 1] = b.y, H0[k + 2] = b.z, H0[k + 3] = b.w;
            if constexpr (PAIR) {
                const float4 c = *reinterpret_cast<const float4 *>(bl + k), d = *reinterpret_cast<const float4 *>(bh + k);
                L1[k] = c.x, L1[k + 1] = c.y, L1[k + 2] = c.z, L1[k + 3] = c.w;
                H1[k] = d.x, H1[k + 1] = d.y, H1[k + 2] = d.z, H1[k + 3] = d.w;
            }
        }
#pragma unroll
        for (int k = 0; k < SEGN / 2; k++) {
            if constexpr (PAIR) {
                v[2 * k] = f2(L0[k + 2], L1[k + 2]);
                v[2 * k + 1] = f2(H0[k + 2], H1[k + 2]);
            } else {
                v[2 * k] = L0[k + 2];
                v[2 * k + 1] = H0[k + 2];
            }
        }
    }
    __syncthreads();  // neighbouring segments overlap: every read before any write
    if constexpr (PAIR) lift2<SEGN>(v);
    else lift1<SEGN>(v);
    // outputs v[4 .. 36): band columns j0 + 2 .. j0 + 18, four at a time
    float *al = band_row(c0, r, 0) + j0 + 2, *ah = band_row(c0, r, 1) + j0 + 2;
    float *bl = band_row(c1, r, 0) + j0 + 2, *bh = band_row(c1, r, 1) + j0 + 2;
#pragma unroll
    for (int k = 0; k < SEG / 2; k += 4) {
        const int o = H + 2 * k;
        if constexpr (PAIR) {
            *reinterpret_cast<float4 *>(al + k) = make_float4(v[o].x, v[o + 2].x, v[o + 4].x, v[o + 6].x);
            *reinterpret_cast<float4 *>(ah + k) = make_float4(v[o + 1].x, v[o + 3].x, v[o + 5].x, v[o + 7].x);
            *reinterpret_cast<float4 *>(bl + k) = make_float4(v[o].y, v[o + 2].y, v[o + 4].y, v[o + 6].y);
            *reinterpret_cast<float4 *>(bh + k) = make_float4(v[o + 1].y, v[o + 3].y, v[o + 5].y, v[o + 7].y);
        } else {
            *reinterpret_cast<float4 *>(al + k) = make_float4(v[o], v[o + 2], v[o + 4], v[o + 6]);
            *reinterpret_cast<float4 *>(ah + k) = make_float4(v[o + 1], v[o + 3], v[o + 5], v[o + 7]);
        }
    }
}

// Rebuilds the extended tile's cells outside the plane (within 4 of its
// border) by whole-sample symmetric extension: columns first (every row),
// then whole rows, so the corners come out right.
__device__ __forceinline__ void extend_borders(float *comps, int x0, int y0, int w, int h)
{
    const int tid = threadIdx.x;
    // columns: x in [-4, 0) and [w, w + 4) that fall inside the extended tile
    for (int idx = tid; idx < NR * 8; idx += kThreads) {
        const int r = idx >> 3, k = idx & 7;
        const int x = k < 4 ? k - 4 : w + (k - 4);
        const int e = x - x0 + H;
        if (e < 0 || e >= TX + 2 * H || (k < 4 && x0 != 0)) continue;
        const int es = mirror(x, w) - x0 + H;
#pragma unroll
        for (int c = 0; c < 3; c++) cell(comps + c * COMPF, r, e) = cell(comps + c * COMPF, r, es);
    }
    __syncthreads();
    // rows: y in [-4, 0) and [h, h + 4) inside the tile, copied whole
    for (int idx = tid; idx < 8 * 2 * BW * 3; idx += kThreads) {
        const int j = idx % BW, p = (idx / BW) & 1, k = (idx / (2 * BW)) & 7, c = idx / (16 * BW);
        const int y = k < 4 ? k - 4 : h + (k - 4);
        const int r = y - y0 + H;
        if (r < 0 || r >= NR || (k < 4 && y0 != 0)) continue;
        const int rs = mirror(y, h) - y0 + H;
        float *comp = comps + c * COMPF;
        band_row(comp, r, p)[j] = band_row(comp, rs, p)[j];
    }
    __syncthreads();
}

// Thread 0: the twelve box copies of tile (bx, by) onto `bar`.
__device__ __forceinline__ void issue_tile(const IctMaps &maps, float *comps, uint32_t bar, int bx, int by, int wl,
                                           int hl)
{
    // order this CTA's earlier shared-memory accesses (generic proxy) before
    // the copies' writes (async proxy) into the same buffer
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, kTileBytes);
    const int xl = bx * (TX / 2) - 4, yl = by * (TY / 2) - 2;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const uint32_t base = smem_addr(comps + c * COMPF);
        tma_load_2d(base + 0 * kBoxBytes, &maps.ll[c], xl, yl, bar);
        tma_load_2d(base + 1 * kBoxBytes, &maps.coef[c], wl + xl, yl, bar);
        tma_load_2d(base + 2 * kBoxBytes, &maps.coef[c], xl, hl + yl, bar);
        tma_load_2d(base + 3 * kBoxBytes, &maps.coef[c], wl + xl, hl + yl, bar);
    }
}

// Persistent CTAs (two per SM) walk the tiles t = blockIdx.x, blockIdx.x +
// gridDim.x, ...  Once the vertical pass has read its columns into
// registers the staging buffer is free, and thread 0 starts the next tile's
// copies, which land while this tile is lifted, colour-transformed and
// stored.
template <typename OT>
__global__ void __launch_bounds__(kThreads, 2)
    idwt97_ict_tma_kernel(const __grid_constant__ IctMaps maps, TileArgs a, uint32_t *err, int ntx, int ntiles)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float *comps = reinterpret_cast<float *>(smem_raw);
    const uint32_t bar = smem_addr(smem_raw + (size_t)3 * COMPF * 4);
    const int tid = threadIdx.x;
    const int w = a.w, h = a.h, wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    float *Y = comps, *Cb = comps + COMPF, *Cr = comps + 2 * COMPF;
    // Vertical pass: warp w takes one half of the rows (w / 4) and 32
    // columns of one parity (w & 1: the low or the high band array), so its
    // lanes read 32 consecutive cells of one array, free of bank conflicts.
    const int vw = tid >> 5, lane = tid & 31;
    const int half = vw >> 2, p = vw & 1, col = 64 * ((vw >> 1) & 1) + 2 * lane + p;
    const int vbase = half ? 32 - H : 0, obase = half ? OUTR : 0;
    const int j = (col >> 1) + 4;   // band column of extended column col + 4
    const float fa = sf_factor(0, p, true, true), fb = sf_factor(1, p, true, true);  // obase and y0 are even
    const OutRange R = out_range(a.bits);
    const bool sgn = a.bits & TC_SIGNED;
    const float dc = (float)R.dc;

    pdl_allow_next();
    if (tid == 0) mbar_init(bar, 1);
    __syncthreads();
    pdl_wait_prev();   // the LL input is the previous level's output
    int t = blockIdx.x;
    if (t >= ntiles) return;
    if (tid == 0) issue_tile(maps, comps, bar, t % ntx, t / ntx, wl, hl);
    uint32_t phase = 0;
    for (; t < ntiles; t += gridDim.x) {
        const int bx = t % ntx, by = t / ntx, x0 = bx * TX, y0 = by * TY;
        // every thread waits (bounded); all leave together if any gave up
        const bool landed = mbar_wait(bar, phase);
        if (__syncthreads_or(!landed)) {
            if (tid == 0) atomicOr(err, TC_DERR_TIMEOUT);
            return;
        }
        phase ^= 1u;
        const bool interior = x0 >= H && x0 + TX + H <= w && y0 >= H && y0 + NR - H <= h;
        if (!interior) extend_borders(comps, x0, y0, w, h);
        hpass<true>(Y, Cb, tid & 63, tid >> 6);
        hpass<false>(Cr, Cr, tid & 63, tid >> 6);
        __syncthreads();

        float2 yc[OUTR];
        {
            float2 v[VN];
#pragma unroll
            for (int k = 0; k < VN; k++) v[k] = f2(band_row(Y, vbase + k, p)[j], band_row(Cb, vbase + k, p)[j]);
            lift2<VN>(v);
#pragma unroll
            for (int r = 0; r < OUTR; r++) yc[r] = v[H + r];
        }
        float u[VN];
#pragma unroll
        for (int k = 0; k < VN; k++) u[k] = band_row(Cr, vbase + k, p)[j];
        __syncthreads();   // every read of this tile is done: the buffer takes the next one
        if (tid == 0 && t + (int)gridDim.x < ntiles) {
            const int tn = t + gridDim.x;
            issue_tile(maps, comps, bar, tn % ntx, tn / ntx, wl, hl);
        }
        lift1<VN>(u);
        const int x = x0 + col, y = y0 + obase;
        if (x < w) {
            const bool full = y + OUTR <= h;
            const size_t o = (size_t)y * a.out_pitch + x;
            OT *o0 = static_cast<OT *>(a.out[0]) + o, *o1 = static_cast<OT *>(a.out[1]) + o,
               *o2 = static_cast<OT *>(a.out[2]) + o;
#pragma unroll
            for (int r = 0; r < OUTR; r++) {
                if (!(full || y + r < h)) continue;
                const float f = (r & 1) ? fb : fa;
                const float Yv = yc[r].x, Cbv = yc[r].y, Crv = u[H + r];
                const float yf = fmaf(f, Yv, dc);
                const float Rc = fmaf(1.402f * f, Crv, yf);
                const float Gc = fmaf(-0.71414f * f, Crv, fmaf(-0.34413f * f, Cbv, yf));
                const float B = fmaf(1.772f * f, Cbv, yf);
                const size_t ro = (size_t)r * a.out_pitch;
                o0[ro] = to_out<OT>(Rc, R, sgn);
                o1[ro] = to_out<OT>(Gc, R, sgn);
                o2[ro] = to_out<OT>(B, R, sgn);
            }
        }
    }
}

// ---- host --------------------------------------------------------------------

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn()
{
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// A 2-D float tensor map of `cols` x `rows` at base with a row pitch of
// pitch_elems, boxes of BW x BR.
bool make_map(CUtensorMap *m, const void *base, int cols, int rows, int pitch_elems)
{
    EncodeTiled fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dim[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t stride[1] = {(cuuint64_t)pitch_elems * 4};
    const cuuint32_t box[2] = {(cuuint32_t)BW, (cuuint32_t)BR};
    const cuuint32_t estride[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dim, stride, box, estride,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace

bool rev97_tma_handles(const LevelIO &io, int out_type)
{
    const int wl = (io.w + 1) >> 1;
    if (io.ncomp != 3 || (out_type != TC_U8 && out_type != TC_U16) || io.w < 16 || io.h < 16) return false;
    if ((wl & 3) || (io.ll_pitch & 3) || (io.coef_pitch & 3)) return false;
    for (int c = 0; c < 3; c++)
        if (!aligned16(io.ll[c]) || !aligned16(io.coef[c])) return false;
    return encode_fn() != nullptr;
}

cudaError_t launch_rev97_tma(tc_ctx *ctx, const LevelIO &io, int out_type, int bits)
{
    IctMaps maps;
    const int wl = (io.w + 1) >> 1, hl = (io.h + 1) >> 1;
    for (int c = 0; c < 3; c++)
        if (!make_map(&maps.ll[c], io.ll[c], wl, hl, io.ll_pitch) ||
            !make_map(&maps.coef[c], io.coef[c], io.w, io.h, io.coef_pitch))
            return cudaErrorInvalidValue;
    TileArgs a;
    a.w = io.w;
    a.h = io.h;
    a.out_pitch = io.out_pitch;
    a.bits = bits;
    for (int c = 0; c < 3; c++) a.out[c] = io.out[c];
    const int ntx = (io.w + TX - 1) / TX, ntiles = ntx * ((io.h + TY - 1) / TY);
    // two persistent CTAs per SM (the shared memory of one tile each)
    const dim3 grid(std::min(ntiles, 2 * num_sms(ctx->device)));
    cudaError_t e;
    if (out_type == TC_U8) {
        static DeviceFlags attr;
        if ((e = set_smem_once(attr, ctx->device, idwt97_ict_tma_kernel<uint8_t>, kSmem)) != cudaSuccess) return e;
        e = launch_pdl(idwt97_ict_tma_kernel<uint8_t>, grid, dim3(kThreads), kSmem, ctx->stream, maps, a,
                       ctx->d_words, ntx, ntiles);
    } else {
        static DeviceFlags attr;
        if ((e = set_smem_once(attr, ctx->device, idwt97_ict_tma_kernel<uint16_t>, kSmem)) != cudaSuccess) return e;
        e = launch_pdl(idwt97_ict_tma_kernel<uint16_t>, grid, dim3(kThreads), kSmem, ctx->stream, maps, a,
                       ctx->d_words, ntx, ntiles);
    }
    ctx->launches++;
    return e;
}

}  // namespace tc
