// dwt_rev97.cu -- the last reverse 9/7 level of a three-component image
// with the inverse ICT fused in, for sm_100a, with packed fp32x2 lifting.
//
// A 256-thread CTA reconstructs one 128 x 56 output tile of all three
// components.  Y and Cb share shared-memory cells of two floats, so every
// lifting step works on both with one FADD2 + one FFMA2 (the packed fp32x2
// instructions of sm_100); Cr has a tile of its own.  The vertical pass
// keeps the Y/Cb column in registers while it lifts the Cr column, so no
// component is parked in shared memory, and the colour transform, DC shift,
// rounding and saturation follow in registers (the reference's tci_kernel
// and idc_level_shift_kernel, Preprocessor.cpp:44-180).
//
// The lifting is scaling-free (dwt_common.cuh): the per-parity factor of
// the two passes is folded into the colour transform's coefficients.  Rows
// first, then columns (2D_SR).  Staging is as in dwt_rev.cu: the 64 x 136
// extended tile (a halo of 4, whole-sample symmetric extension of ISO
// F.3.7) is copied with 4-byte asynchronous copies straight from the four
// Mallat subbands; for the paired tile a half-warp fills the Y row and the
// other half the Cb row.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "dwt_common.cuh"
#include "tc_internal.cuh"

namespace tc {
namespace {

using namespace dwt;

constexpr int kThreads = 256;
constexpr int H = 4, NR = 64, TY = NR - 2 * H, TX = 128, NC = TX + 2 * H;
constexpr int S2 = NC + 2;  // float2 cells per row: S2/2 odd (16-byte row accesses spread over the banks)
constexpr int S1 = NC + 4;  // floats per row of a single tile: S1/4 odd
static_assert((S2 / 2) % 2 == 1 && (S1 / 4) % 2 == 1, "row strides");
constexpr int SEG = 32, SEGN = SEG + 2 * H;


__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// In-place scaling-free reverse 9/7 lifting of an interleaved signal (v[0]
// at an even position).  Samples at least H from both ends are exact.
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

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Round to nearest even, saturate to the output type's range and clamp to
// [R.lo, R.hi] when the samples are narrower than the type; signed samples
// are stored in two's complement.
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

// Stages component `comp`'s 64 x 136 extended window of tile (bx, by) into
// the float slots dst[r * rs + e * es] (rs, es in floats); each half-warp
// copies whole rows, 16 elements per copy instruction.
__device__ __forceinline__ void stage(const LevelIO &io, int comp, int bx, int by, float *dst, int rs, int es)
{
    const float *ll = static_cast<const float *>(io.ll[comp]);
    const float *coef = static_cast<const float *>(io.coef[comp]);
    const int w = io.w, h = io.h, wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    const int x0 = bx * TX, y0 = by * TY;
    const int hl16 = threadIdx.x & 15, warp = threadIdx.x >> 5;
    const bool interior = x0 >= H && x0 + TX + H <= w && y0 >= H && y0 + NR - H <= h;
    if (interior) {
        // x0 - H is even: element e of a row is band (e & 1) at index
        // (x0 - H + e) / 2, so a lane's sources are one stride-8 run
        const int xs = ((x0 - H) >> 1) + (hl16 >> 1);
        for (int r = warp; r < NR; r += kThreads / 32) {
            const int y = y0 - H + r, yb = y >> 1;
            const float *src = (y & 1) ? coef + (size_t)(hl + yb) * io.coef_pitch + ((hl16 & 1) ? wl : 0)
                                       : ((hl16 & 1) ? coef + (size_t)yb * io.coef_pitch + wl
                                                     : ll + (size_t)yb * io.ll_pitch);
            src += xs;
            float *d = dst + r * rs + hl16 * es;
#pragma unroll
            for (int j = 0; j < NC / 16; j++) cp_async4(d + 16 * j * es, src + 8 * j);
            if (hl16 < NC % 16) cp_async4(d + 16 * (NC / 16) * es, src + 8 * (NC / 16));
        }
    } else {
        for (int r = warp; r < NR; r += kThreads / 32) {
            const int my = mirror(y0 - H + r, h), yb = my >> 1;
            const float *lrow = (my & 1) ? coef + (size_t)(hl + yb) * io.coef_pitch : ll + (size_t)yb * io.ll_pitch;
            const float *hrow = coef + (size_t)((my & 1) ? hl + yb : yb) * io.coef_pitch + wl;
#pragma unroll
            for (int e = hl16; e < NC; e += 16) {
                const int mx = mirror(x0 - H + e, w);
                cp_async4(dst + r * rs + e * es, ((mx & 1) ? hrow : lrow) + (mx >> 1));
            }
        }
    }
}

// Horizontal pass over the paired tile: thread (seg, r) lifts one 32-output
// segment of row r of both components.
__device__ __forceinline__ void hpass2(float2 *t2)
{
    const int tid = threadIdx.x, seg = tid / NR, r = tid % NR;
    float2 *row = t2 + r * S2 + seg * SEG;
    float2 v[SEGN];
#pragma unroll
    for (int k = 0; k < SEGN; k += 2) {
        const float4 q = *reinterpret_cast<const float4 *>(row + k);
        v[k] = f2(q.x, q.y);
        v[k + 1] = f2(q.z, q.w);
    }
    __syncthreads();  // neighbouring segments overlap: all reads before any write
    lift2<SEGN>(v);
#pragma unroll
    for (int k = H; k < H + SEG; k += 2)
        *reinterpret_cast<float4 *>(row + k) = make_float4(v[k].x, v[k].y, v[k + 1].x, v[k + 1].y);
}

__device__ __forceinline__ void hpass1(float *t1)
{
    const int tid = threadIdx.x, seg = tid / NR, r = tid % NR;
    float *row = t1 + r * S1 + seg * SEG;
    float v[SEGN];
#pragma unroll
    for (int k = 0; k < SEGN; k += 4) {
        const float4 q = *reinterpret_cast<const float4 *>(row + k);
        v[k] = q.x;
        v[k + 1] = q.y;
        v[k + 2] = q.z;
        v[k + 3] = q.w;
    }
    __syncthreads();
    lift1<SEGN>(v);
#pragma unroll
    for (int k = H; k < H + SEG; k += 4)
        *reinterpret_cast<float4 *>(row + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
}

// Vertical pass geometry: two threads per column; the top one lifts tile
// rows [0, 32 + H) and keeps output rows [0, 32 - H), the bottom one lifts
// [32 - H, 64) and keeps [32 - H, TY).
constexpr int VN = 32 + H, OUTR = 32 - H;

// Inverse-ICT last level of one image tile: Y and Cb paired, Cr single.
template <typename OT>
__device__ __forceinline__ void ict_tile(const LevelIO &io, int bx, int by, int bits)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *t2 = reinterpret_cast<float2 *>(smem_raw);
    float *tf = reinterpret_cast<float *>(smem_raw);
    float *t1 = tf + 2 * NR * S2;
    const int tid = threadIdx.x;
    const int sub = (tid >> 4) & 1;
    // Y into the .x slots, Cb into .y (a half-warp each)
    stage(io, sub, bx, by, tf + sub, 2 * S2, 2);
    // Cr: staged by whole warps into the single-tile layout
    {
        const float *ll = static_cast<const float *>(io.ll[2]);
        const float *coef = static_cast<const float *>(io.coef[2]);
        const int w = io.w, h = io.h, wl = (w + 1) >> 1, hl = (h + 1) >> 1;
        const int x0 = bx * TX, y0 = by * TY, lane = tid & 31, warp = tid >> 5;
        const bool interior = x0 >= H && x0 + TX + H <= w && y0 >= H && y0 + NR - H <= h;
        if (interior) {
            const int xs = ((x0 - H) >> 1) + (lane >> 1);
            for (int r = warp; r < NR; r += kThreads / 32) {
                const int y = y0 - H + r, yb = y >> 1;
                const float *src = (y & 1) ? coef + (size_t)(hl + yb) * io.coef_pitch + ((lane & 1) ? wl : 0)
                                           : ((lane & 1) ? coef + (size_t)yb * io.coef_pitch + wl
                                                         : ll + (size_t)yb * io.ll_pitch);
                src += xs;
                float *d = t1 + r * S1 + lane;
#pragma unroll
                for (int j = 0; j < NC / 32; j++) cp_async4(d + 32 * j, src + 16 * j);
                if (lane < NC % 32) cp_async4(d + 32 * (NC / 32), src + 16 * (NC / 32));
            }
        } else {
            for (int r = warp; r < NR; r += kThreads / 32) {
                const int my = mirror(y0 - H + r, h), yb = my >> 1;
                const float *lrow =
                    (my & 1) ? coef + (size_t)(hl + yb) * io.coef_pitch : ll + (size_t)yb * io.ll_pitch;
                const float *hrow = coef + (size_t)((my & 1) ? hl + yb : yb) * io.coef_pitch + wl;
#pragma unroll
                for (int e = lane; e < NC; e += 32) {
                    const int mx = mirror(x0 - H + e, w);
                    cp_async4(t1 + r * S1 + e, ((mx & 1) ? hrow : lrow) + (mx >> 1));
                }
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();

    const bool hx = io.w > 1, vy = io.h > 1;
    if (hx) {
        hpass2(t2);
        hpass1(t1);
        __syncthreads();
    }

    const int col = tid % TX, half = tid / TX;
    const int vbase = half ? 32 - H : 0, obase = half ? OUTR : 0;
    const int x = bx * TX + col, y = by * TY + obase;
    float2 yc[OUTR];
    {
        float2 v[VN];
#pragma unroll
        for (int k = 0; k < VN; k++) v[k] = t2[(vbase + k) * S2 + H + col];
        if (vy) lift2<VN>(v);
#pragma unroll
        for (int r = 0; r < OUTR; r++) yc[r] = v[H + r];
    }
    float cr[VN];
#pragma unroll
    for (int k = 0; k < VN; k++) cr[k] = t1[(vbase + k) * S1 + H + col];
    if (vy) lift1<VN>(cr);
    if (x >= io.w) return;
    const bool full = y + OUTR <= io.h;
    const int cx = col & 1;
    const float fa = sf_factor(0, cx, hx, vy), fb = sf_factor(1, cx, hx, vy);  // obase is even
    const OutRange R = out_range(bits);
    const bool sgn = bits & TC_SIGNED;
    const float dc = (float)R.dc;
    const size_t o = (size_t)y * io.out_pitch + x;
    OT *o0 = static_cast<OT *>(io.out[0]) + o, *o1 = static_cast<OT *>(io.out[1]) + o,
       *o2 = static_cast<OT *>(io.out[2]) + o;
#pragma unroll
    for (int r = 0; r < OUTR; r++) {
        if (!(full || y + r < io.h)) continue;
        const float f = (r & 1) ? fb : fa;
        const float Y = yc[r].x, Cb = yc[r].y, Cr = cr[H + r];
        // inverse ICT (ISO G.3) on the unscaled samples, the output factor
        // and the DC shift folded into the coefficients
        const float yf = fmaf(f, Y, dc);
        const float Rc = fmaf(1.402f * f, Cr, yf);
        const float Gc = fmaf(-0.71414f * f, Cr, fmaf(-0.34413f * f, Cb, yf));
        const float B = fmaf(1.772f * f, Cb, yf);
        const size_t ro = (size_t)r * io.out_pitch;
        o0[ro] = to_out<OT>(Rc, R, sgn);
        o1[ro] = to_out<OT>(Gc, R, sgn);
        o2[ro] = to_out<OT>(B, R, sgn);
    }
}

// ---- kernels ------------------------------------------------------------------

template <typename OT>
__global__ void __launch_bounds__(kThreads, 2) idwt97_ict_kernel(LevelIO io, int bits)
{
    pdl_allow_next();
    pdl_wait_prev();
    ict_tile<OT>(io, blockIdx.x, blockIdx.y, bits);
}

template <typename OT>
__global__ void __launch_bounds__(kThreads, 2) idwt97_ict_batch_kernel(const RevJob *__restrict__ jobs, int njobs,
                                                                      int bits)
{
    pdl_allow_next();
    const int b = blockIdx.x;
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].tile0 <= b) lo = mid;
        else hi = mid - 1;
    }
    const RevJob &J = jobs[lo];
    const int t = b - J.tile0;
    pdl_wait_prev();
    ict_tile<OT>(J.io, t % J.tiles_x, t / J.tiles_x, bits);
}

constexpr size_t kIctSmem = (size_t)NR * S2 * sizeof(float2) + (size_t)NR * S1 * sizeof(float);

template <typename OT>
cudaError_t ict_level(tc_ctx *ctx, const LevelIO &io, int bits)
{
    static DeviceFlags attr;
    cudaError_t e = set_smem_once(attr, ctx->device, idwt97_ict_kernel<OT>, kIctSmem);
    if (e != cudaSuccess) return e;
    dim3 grid((io.w + TX - 1) / TX, (io.h + TY - 1) / TY);
    e = launch_pdl(idwt97_ict_kernel<OT>, grid, dim3(kThreads), kIctSmem, ctx->stream, io, bits);
    ctx->launches++;
    return e;
}

template <typename OT>
cudaError_t ict_batch(tc_ctx *ctx, const RevJob *jobs, int njobs, int ntiles, int bits)
{
    static DeviceFlags attr;
    cudaError_t e = set_smem_once(attr, ctx->device, idwt97_ict_batch_kernel<OT>, kIctSmem);
    if (e != cudaSuccess) return e;
    e = launch_pdl(idwt97_ict_batch_kernel<OT>, dim3(ntiles), dim3(kThreads), kIctSmem, ctx->stream, jobs, njobs,
                   bits);
    ctx->launches++;
    return e;
}

}  // namespace

bool rev97_handles(int color, int ncomp, int out_type)
{
    return color == TC_COLOR_ICT && ncomp == 3 && (out_type == TC_U8 || out_type == TC_U16);
}

cudaError_t launch_rev97_level(tc_ctx *ctx, const LevelIO &io, int out_type, int bits)
{
    if (io.w <= 0 || io.h <= 0) return cudaSuccess;
    return out_type == TC_U8 ? ict_level<uint8_t>(ctx, io, bits) : ict_level<uint16_t>(ctx, io, bits);
}

cudaError_t launch_rev97_batch(tc_ctx *ctx, const RevJob *d_jobs, int njobs, int ntiles, int out_type, int bits)
{
    if (njobs <= 0 || ntiles <= 0) return cudaSuccess;
    return out_type == TC_U8 ? ict_batch<uint8_t>(ctx, d_jobs, njobs, ntiles, bits)
                             : ict_batch<uint16_t>(ctx, d_jobs, njobs, ntiles, bits);
}

}  // namespace tc
