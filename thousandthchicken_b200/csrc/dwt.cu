// dwt.cu -- 5/3 (int32) and 9/7 (fp32) lifting DWT levels for sm_100a.
//
// Replaces the reference's sliding-window kernels (dwt_r53.cl, dwt_r97.cl,
// dwt_f53.cl, dwt_f97.cl over dwt_transform_buffer.cl / dwt_io.cl) and the
// per-level LL copy of DWTKernel::copyLLBandToSrc (DWTKernel.cpp:127-154):
//   * one launch per level; each CTA owns a TX x TY output tile and stages
//     the tile plus a halo of H samples (2 for 5/3, 4 for 9/7) in shared
//     memory, loading straight from the four Mallat subbands with
//     whole-sample symmetric extension (full periodic reflection, ISO F.3.7,
//     instead of the single reflection of dwt_io.cl:7-38, defect D14);
//   * rows are stored split into even/odd halves so every lifting step is a
//     unit-stride, bank-conflict-free sweep; the LL input of a level is read
//     from the previous level's output buffer, so no LL copy is needed;
//   * 5/3 uses floor (ISO) or truncating (reference, defect D13) rounding;
//     9/7 uses fp32 with the scaling factors applied as floats (defects
//     D10-D12 fixed);
//   * the last reverse level can fuse the inverse RCT/ICT, DC shift,
//     rounding and clamp (tcr_kernel / tci_kernel / idc_level_shift_kernel)
//     into its store, writing 8- or 16-bit samples.
#include <cuda_runtime.h>

#include "tc_internal.cuh"

namespace tc {
namespace {

__device__ __forceinline__ int pse(int i, int n)
{
    if (n == 1) return 0;
    const int per = 2 * (n - 1);
    i %= per;
    if (i < 0) i += per;
    return i >= n ? per - i : i;
}

// Index inside [0, n) after extension; the modulo path only runs at borders.
__device__ __forceinline__ int mirror(int i, int n)
{
    return (unsigned)i < (unsigned)n ? i : pse(i, n);
}

// 9/7 lifting constants (ISO F.4.8.2).
constexpr float kA = -1.586134342059924f, kB = -0.052980118572961f, kG = 0.882911075530934f,
                kD = 0.443506852043971f, kK = 1.230174104914001f, kInvK = 1.0f / 1.230174104914001f;

template <int RND>
__device__ __forceinline__ int div4r(int v)
{
    return RND == TC_ROUND_TRUNC ? v / 4 : (v >> 2);
}
template <int RND>
__device__ __forceinline__ int div2r(int v)
{
    return RND == TC_ROUND_TRUNC ? v / 2 : (v >> 1);
}

// A tile buffer of NR rows x NC columns, each row split into an even half
// [0, NC/2) and an odd half [NC/2, NC).
template <typename T, int NR, int NC>
struct Tile {
    static constexpr int NE = NC / 2;
    T d[NR * NC];
    __device__ __forceinline__ T &at(int r, int e) { return d[r * NC + ((e & 1) ? NE + (e >> 1) : (e >> 1))]; }
    __device__ __forceinline__ T &ev(int r, int i) { return d[r * NC + i]; }
    __device__ __forceinline__ T &od(int r, int i) { return d[r * NC + NE + i]; }
};

// ---- horizontal lifting over all rows; vertical over central columns -----

template <typename T, int NR, int NC, int RND>
__device__ void lift_h_rev53(Tile<T, NR, NC> &t)
{
    constexpr int NE = NC / 2;
    for (int q = threadIdx.x; q < NR * (NE - 1); q += blockDim.x) {
        const int r = q / (NE - 1), i = 1 + q % (NE - 1);
        t.ev(r, i) -= div4r<RND>(t.od(r, i - 1) + t.od(r, i) + 2);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NR * (NE - 1); q += blockDim.x) {
        const int r = q / (NE - 1), i = q % (NE - 1);
        t.od(r, i) += div2r<RND>(t.ev(r, i) + t.ev(r, i + 1));
    }
    __syncthreads();
}

template <typename T, int NR, int NC, int RND>
__device__ void lift_v_rev53(Tile<T, NR, NC> &t, int c0, int c1)
{
    // rows 2i (low) and 2i+1 (high); columns [c0, c1) in extended coordinates
    const int ncol = c1 - c0;
    for (int q = threadIdx.x; q < (NR / 2 - 1) * ncol; q += blockDim.x) {
        const int i = 1 + q / ncol, e = c0 + q % ncol;
        t.at(2 * i, e) -= div4r<RND>(t.at(2 * i - 1, e) + t.at(2 * i + 1, e) + 2);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2 - 1) * ncol; q += blockDim.x) {
        const int i = q / ncol, e = c0 + q % ncol;
        t.at(2 * i + 1, e) += div2r<RND>(t.at(2 * i, e) + t.at(2 * i + 2, e));
    }
    __syncthreads();
}

template <int NR, int NC>
__device__ void lift_h_rev97(Tile<float, NR, NC> &t)
{
    constexpr int NE = NC / 2;
    for (int q = threadIdx.x; q < NR * NE; q += blockDim.x) {
        const int r = q / NE, i = q % NE;
        t.ev(r, i) *= kK;
        t.od(r, i) *= kInvK;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NR * (NE - 1); q += blockDim.x) {
        const int r = q / (NE - 1), i = 1 + q % (NE - 1);
        t.ev(r, i) = fmaf(-kD, t.od(r, i - 1) + t.od(r, i), t.ev(r, i));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NR * (NE - 1); q += blockDim.x) {
        const int r = q / (NE - 1), i = q % (NE - 1);
        t.od(r, i) = fmaf(-kG, t.ev(r, i) + t.ev(r, i + 1), t.od(r, i));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NR * (NE - 1); q += blockDim.x) {
        const int r = q / (NE - 1), i = 1 + q % (NE - 1);
        t.ev(r, i) = fmaf(-kB, t.od(r, i - 1) + t.od(r, i), t.ev(r, i));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NR * (NE - 1); q += blockDim.x) {
        const int r = q / (NE - 1), i = q % (NE - 1);
        t.od(r, i) = fmaf(-kA, t.ev(r, i) + t.ev(r, i + 1), t.od(r, i));
    }
    __syncthreads();
}

template <int NR, int NC>
__device__ void lift_v_rev97(Tile<float, NR, NC> &t, int c0, int c1)
{
    const int ncol = c1 - c0;
    for (int q = threadIdx.x; q < (NR / 2) * ncol; q += blockDim.x) {
        const int i = q / ncol, e = c0 + q % ncol;
        t.at(2 * i, e) *= kK;
        t.at(2 * i + 1, e) *= kInvK;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2 - 1) * ncol; q += blockDim.x) {
        const int i = 1 + q / ncol, e = c0 + q % ncol;
        t.at(2 * i, e) = fmaf(-kD, t.at(2 * i - 1, e) + t.at(2 * i + 1, e), t.at(2 * i, e));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2 - 1) * ncol; q += blockDim.x) {
        const int i = q / ncol, e = c0 + q % ncol;
        t.at(2 * i + 1, e) = fmaf(-kG, t.at(2 * i, e) + t.at(2 * i + 2, e), t.at(2 * i + 1, e));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2 - 1) * ncol; q += blockDim.x) {
        const int i = 1 + q / ncol, e = c0 + q % ncol;
        t.at(2 * i, e) = fmaf(-kB, t.at(2 * i - 1, e) + t.at(2 * i + 1, e), t.at(2 * i, e));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2 - 1) * ncol; q += blockDim.x) {
        const int i = q / ncol, e = c0 + q % ncol;
        t.at(2 * i + 1, e) = fmaf(-kA, t.at(2 * i, e) + t.at(2 * i + 2, e), t.at(2 * i + 1, e));
    }
    __syncthreads();
}

// Forward lifting: vertical over all columns first, then horizontal over
// central rows (ISO F.4.2 order).
template <typename T, int NR, int NC, int RND>
__device__ void lift_v_fwd53(Tile<T, NR, NC> &t)
{
    for (int q = threadIdx.x; q < (NR / 2 - 1) * NC; q += blockDim.x) {
        const int i = q / NC, e = q % NC;
        t.at(2 * i + 1, e) -= div2r<RND>(t.at(2 * i, e) + t.at(2 * i + 2, e));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2 - 2) * NC; q += blockDim.x) {
        const int i = 1 + q / NC, e = q % NC;
        t.at(2 * i, e) += div4r<RND>(t.at(2 * i - 1, e) + t.at(2 * i + 1, e) + 2);
    }
    __syncthreads();
}

template <typename T, int NR, int NC, int RND>
__device__ void lift_h_fwd53(Tile<T, NR, NC> &t, int r0, int r1)
{
    constexpr int NE = NC / 2;
    const int nr = r1 - r0;
    for (int q = threadIdx.x; q < nr * (NE - 1); q += blockDim.x) {
        const int r = r0 + q / (NE - 1), i = q % (NE - 1);
        t.od(r, i) -= div2r<RND>(t.ev(r, i) + t.ev(r, i + 1));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nr * (NE - 2); q += blockDim.x) {
        const int r = r0 + q / (NE - 2), i = 1 + q % (NE - 2);
        t.ev(r, i) += div4r<RND>(t.od(r, i - 1) + t.od(r, i) + 2);
    }
    __syncthreads();
}

template <int NR, int NC>
__device__ void lift_v_fwd97(Tile<float, NR, NC> &t)
{
    for (int q = threadIdx.x; q < (NR / 2 - 1) * NC; q += blockDim.x) {
        const int i = q / NC, e = q % NC;
        t.at(2 * i + 1, e) = fmaf(kA, t.at(2 * i, e) + t.at(2 * i + 2, e), t.at(2 * i + 1, e));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2 - 2) * NC; q += blockDim.x) {
        const int i = 1 + q / NC, e = q % NC;
        t.at(2 * i, e) = fmaf(kB, t.at(2 * i - 1, e) + t.at(2 * i + 1, e), t.at(2 * i, e));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2 - 2) * NC; q += blockDim.x) {
        const int i = 1 + q / NC, e = q % NC;
        t.at(2 * i + 1, e) = fmaf(kG, t.at(2 * i, e) + t.at(2 * i + 2, e), t.at(2 * i + 1, e));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2 - 3) * NC; q += blockDim.x) {
        const int i = 2 + q / NC, e = q % NC;
        t.at(2 * i, e) = fmaf(kD, t.at(2 * i - 1, e) + t.at(2 * i + 1, e), t.at(2 * i, e));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (NR / 2) * NC; q += blockDim.x) {
        const int i = q / NC, e = q % NC;
        t.at(2 * i + 1, e) *= kK;
        t.at(2 * i, e) *= kInvK;
    }
    __syncthreads();
}

template <int NR, int NC>
__device__ void lift_h_fwd97(Tile<float, NR, NC> &t, int r0, int r1)
{
    constexpr int NE = NC / 2;
    const int nr = r1 - r0;
    for (int q = threadIdx.x; q < nr * (NE - 1); q += blockDim.x) {
        const int r = r0 + q / (NE - 1), i = q % (NE - 1);
        t.od(r, i) = fmaf(kA, t.ev(r, i) + t.ev(r, i + 1), t.od(r, i));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nr * (NE - 2); q += blockDim.x) {
        const int r = r0 + q / (NE - 2), i = 1 + q % (NE - 2);
        t.ev(r, i) = fmaf(kB, t.od(r, i - 1) + t.od(r, i), t.ev(r, i));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nr * (NE - 2); q += blockDim.x) {
        const int r = r0 + q / (NE - 2), i = 1 + q % (NE - 2);
        t.od(r, i) = fmaf(kG, t.ev(r, i) + t.ev(r, i + 1), t.od(r, i));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nr * (NE - 3); q += blockDim.x) {
        const int r = r0 + q / (NE - 3), i = 2 + q % (NE - 3);
        t.ev(r, i) = fmaf(kD, t.od(r, i - 1) + t.od(r, i), t.ev(r, i));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nr * NE; q += blockDim.x) {
        const int r = r0 + q / NE, i = q % NE;
        t.od(r, i) *= kK;
        t.ev(r, i) *= kInvK;
    }
    __syncthreads();
}

// ---- loads ---------------------------------------------------------------

// Load the extended reverse tile of one component from the Mallat subbands.
template <typename T, int NR, int NC, int H>
__device__ void load_rev(Tile<T, NR, NC> &t, const T *ll, int llp, const T *coef, int cp, int x0,
                         int y0, int w, int h)
{
    constexpr int NE = NC / 2;
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    for (int q = threadIdx.x; q < NR * NC; q += blockDim.x) {
        const int r = q / NC, rem = q % NC, par = rem / NE, i = rem % NE;
        const int e = 2 * i + par;
        const int my = mirror(y0 - H + r, h), mx = mirror(x0 - H + e, w);
        const int yb = my >> 1, xb = mx >> 1;
        T v;
        if (!(my & 1)) v = (mx & 1) ? coef[(size_t)yb * cp + wl + xb] : ll[(size_t)yb * llp + xb];
        else v = (mx & 1) ? coef[(size_t)(hl + yb) * cp + wl + xb] : coef[(size_t)(hl + yb) * cp + xb];
        t.d[r * NC + (par ? NE : 0) + i] = v;
    }
    __syncthreads();
}

template <typename T, int NR, int NC, int H>
__device__ void load_fwd(Tile<T, NR, NC> &t, const T *in, int ip, int x0, int y0, int w, int h)
{
    constexpr int NE = NC / 2;
    for (int q = threadIdx.x; q < NR * NC; q += blockDim.x) {
        const int r = q / NC, rem = q % NC, par = rem / NE, i = rem % NE;
        const int e = 2 * i + par;
        const int my = mirror(y0 - H + r, h), mx = mirror(x0 - H + e, w);
        t.d[r * NC + (par ? NE : 0) + i] = in[(size_t)my * ip + mx];
    }
    __syncthreads();
}

// ---- kernels --------------------------------------------------------------

template <int WAVELET>
struct Geo {
    static constexpr int H = WAVELET ? 4 : 2;
};

// Reverse level, one component per blockIdx.z, plane output.
template <typename T, int WAVELET, int RND, int TX, int TY>
__global__ void __launch_bounds__(256) idwt_level_kernel(LevelIO io)
{
    constexpr int H = Geo<WAVELET>::H, NR = TY + 2 * H, NC = TX + 2 * H;
    __shared__ Tile<T, NR, NC> t;
    const int c = blockIdx.z;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int w = io.w, h = io.h;
    load_rev<T, NR, NC, H>(t, static_cast<const T *>(io.ll[c]), io.ll_pitch,
                           static_cast<const T *>(io.coef[c]), io.coef_pitch, x0, y0, w, h);
    if constexpr (WAVELET == 0) {
        if (w > 1) lift_h_rev53<T, NR, NC, RND>(t);
        if (h > 1) lift_v_rev53<T, NR, NC, RND>(t, H, H + TX);
    } else {
        if (w > 1) lift_h_rev97<NR, NC>(t);
        if (h > 1) lift_v_rev97<NR, NC>(t, H, H + TX);
    }
    T *out = static_cast<T *>(io.out[c]);
    for (int q = threadIdx.x; q < TX * TY; q += blockDim.x) {
        const int r = q / TX, e = q % TX;
        const int y = y0 + r, x = x0 + e;
        if (y < h && x < w) out[(size_t)y * io.out_pitch + x] = t.at(r + H, e + H);
    }
}

// Forward level, one component per blockIdx.z.
template <typename T, int WAVELET, int RND, int TX, int TY>
__global__ void __launch_bounds__(256) fdwt_level_kernel(LevelIO io)
{
    constexpr int H = Geo<WAVELET>::H, NR = TY + 2 * H, NC = TX + 2 * H;
    __shared__ Tile<T, NR, NC> t;
    const int c = blockIdx.z;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int w = io.w, h = io.h;
    load_fwd<T, NR, NC, H>(t, static_cast<const T *>(io.ll[c]), io.ll_pitch, x0, y0, w, h);
    if constexpr (WAVELET == 0) {
        if (h > 1) lift_v_fwd53<T, NR, NC, RND>(t);
        if (w > 1) lift_h_fwd53<T, NR, NC, RND>(t, H, H + TY);
    } else {
        if (h > 1) lift_v_fwd97<NR, NC>(t);
        if (w > 1) lift_h_fwd97<NR, NC>(t, H, H + TY);
    }
    const int wl = (w + 1) >> 1, hl = (h + 1) >> 1;
    T *ll = static_cast<T *>(io.out[c]);
    T *bands = static_cast<T *>(io.bands[c]);
    constexpr int NE = TX / 2;
    // group stores so a warp writes consecutive elements of one band row
    for (int q = threadIdx.x; q < TX * TY; q += blockDim.x) {
        const int r = q / TX, rem = q % TX, par = rem / NE, i = rem % NE;
        const int e = 2 * i + par;
        const int y = y0 + r, x = x0 + e;
        if (y >= h || x >= w) continue;
        const T v = t.at(r + H, e + H);
        const int yb = y >> 1, xb = x >> 1;
        if (!(y & 1)) {
            if (!(x & 1)) ll[(size_t)yb * io.out_pitch + xb] = v;
            else bands[(size_t)yb * io.bands_pitch + wl + xb] = v;
        } else {
            if (!(x & 1)) bands[(size_t)(hl + yb) * io.bands_pitch + xb] = v;
            else bands[(size_t)(hl + yb) * io.bands_pitch + wl + xb] = v;
        }
    }
}

// ---- last reverse level fused with colour ---------------------------------

template <typename OT>
__device__ __forceinline__ OT clamp_out(int v, int mx)
{
    return (OT)(v < 0 ? 0 : (v > mx ? mx : v));
}

template <typename T, int WAVELET, int RND, int COLOR, typename OT, int NCOMP>
__global__ void __launch_bounds__(256) idwt_last_color_kernel(LevelIO io, int bits)
{
    constexpr int TX = 64, TY = 32;
    constexpr int H = Geo<WAVELET>::H, NR = TY + 2 * H, NC = TX + 2 * H;
    constexpr int PER = TX * TY / 256;
    __shared__ Tile<T, NR, NC> t;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int w = io.w, h = io.h;
    T res[NCOMP][PER];
#pragma unroll
    for (int c = 0; c < NCOMP; c++) {
        if (c) __syncthreads();
        load_rev<T, NR, NC, H>(t, static_cast<const T *>(io.ll[c]), io.ll_pitch,
                               static_cast<const T *>(io.coef[c]), io.coef_pitch, x0, y0, w, h);
        if constexpr (WAVELET == 0) {
            if (w > 1) lift_h_rev53<T, NR, NC, RND>(t);
            if (h > 1) lift_v_rev53<T, NR, NC, RND>(t, H, H + TX);
        } else {
            if (w > 1) lift_h_rev97<NR, NC>(t);
            if (h > 1) lift_v_rev97<NR, NC>(t, H, H + TX);
        }
#pragma unroll
        for (int j = 0; j < PER; j++) {
            const int q = threadIdx.x + 256 * j;
            res[c][j] = t.at(q / TX + H, q % TX + H);
        }
    }
    const int dc = 1 << (bits - 1), mx = (1 << bits) - 1;
#pragma unroll
    for (int j = 0; j < PER; j++) {
        const int q = threadIdx.x + 256 * j;
        const int y = y0 + q / TX, x = x0 + q % TX;
        if (y >= h || x >= w) continue;
        const size_t o = (size_t)y * io.out_pitch + x;
        int v[4];
        if constexpr (COLOR == TC_COLOR_RCT) {
            const int Y = (int)res[0][j], U = (int)res[1][j], V = (int)res[2][j];
            const int G = Y - ((U + V) >> 2);
            v[0] = V + G;
            v[1] = G;
            v[2] = U + G;
        } else if constexpr (COLOR == TC_COLOR_ICT) {
            const float Y = (float)res[0][j], Cb = (float)res[1][j], Cr = (float)res[2][j];
            v[0] = __float2int_rn(fmaf(1.402f, Cr, Y));
            v[1] = __float2int_rn(Y - 0.34413f * Cb - 0.71414f * Cr);
            v[2] = __float2int_rn(fmaf(1.772f, Cb, Y));
        }
#pragma unroll
        for (int c = 0; c < NCOMP; c++) {
            int s;
            if (COLOR != TC_COLOR_DC && c < 3) s = v[c];
            else if constexpr (WAVELET == 0) s = (int)res[c][j];
            else s = __float2int_rn((float)res[c][j]);
            static_cast<OT *>(io.out[c])[o] = clamp_out<OT>(s + dc, mx);
        }
    }
}

template <typename T, int WAVELET, int RND, int TX, int TY>
cudaError_t run_idwt(tc_ctx *ctx, const LevelIO &io)
{
    dim3 grid((io.w + TX - 1) / TX, (io.h + TY - 1) / TY, io.ncomp);
    idwt_level_kernel<T, WAVELET, RND, TX, TY><<<grid, 256, 0, ctx->stream>>>(io);
    ctx->launches++;
    return cudaGetLastError();
}

template <typename T, int WAVELET, int RND, int TX, int TY>
cudaError_t run_fdwt(tc_ctx *ctx, const LevelIO &io)
{
    dim3 grid((io.w + TX - 1) / TX, (io.h + TY - 1) / TY, io.ncomp);
    fdwt_level_kernel<T, WAVELET, RND, TX, TY><<<grid, 256, 0, ctx->stream>>>(io);
    ctx->launches++;
    return cudaGetLastError();
}

template <typename T, int WAVELET, int RND, int COLOR, int NCOMP>
cudaError_t run_last_n(tc_ctx *ctx, const LevelIO &io, int out_type, int bits)
{
    dim3 grid((io.w + 63) / 64, (io.h + 31) / 32, 1);
    if (out_type == TC_U8)
        idwt_last_color_kernel<T, WAVELET, RND, COLOR, uint8_t, NCOMP><<<grid, 256, 0, ctx->stream>>>(io, bits);
    else if (out_type == TC_U16)
        idwt_last_color_kernel<T, WAVELET, RND, COLOR, uint16_t, NCOMP><<<grid, 256, 0, ctx->stream>>>(io, bits);
    else
        idwt_last_color_kernel<T, WAVELET, RND, COLOR, int32_t, NCOMP><<<grid, 256, 0, ctx->stream>>>(io, bits);
    ctx->launches++;
    return cudaGetLastError();
}

template <typename T, int WAVELET, int RND, int COLOR>
cudaError_t run_last(tc_ctx *ctx, const LevelIO &io, int out_type, int bits)
{
    if (COLOR != TC_COLOR_DC) {
        if (io.ncomp == 4) return run_last_n<T, WAVELET, RND, COLOR, 4>(ctx, io, out_type, bits);
        return run_last_n<T, WAVELET, RND, COLOR, 3>(ctx, io, out_type, bits);
    }
    switch (io.ncomp) {
    case 1: return run_last_n<T, WAVELET, RND, COLOR, 1>(ctx, io, out_type, bits);
    case 2: return run_last_n<T, WAVELET, RND, COLOR, 2>(ctx, io, out_type, bits);
    case 3: return run_last_n<T, WAVELET, RND, COLOR, 3>(ctx, io, out_type, bits);
    default: return run_last_n<T, WAVELET, RND, COLOR, 4>(ctx, io, out_type, bits);
    }
}

}  // namespace

cudaError_t launch_idwt_level(tc_ctx *ctx, const LevelIO &io, int wavelet, int rounding)
{
    if (io.w <= 0 || io.h <= 0) return cudaSuccess;
    if (wavelet) return run_idwt<float, 1, 0, 128, 64>(ctx, io);
    if (rounding == TC_ROUND_TRUNC) return run_idwt<int32_t, 0, TC_ROUND_TRUNC, 128, 64>(ctx, io);
    return run_idwt<int32_t, 0, TC_ROUND_FLOOR, 128, 64>(ctx, io);
}

cudaError_t launch_fdwt_level(tc_ctx *ctx, const LevelIO &io, int wavelet, int rounding)
{
    if (io.w <= 0 || io.h <= 0) return cudaSuccess;
    if (wavelet) return run_fdwt<float, 1, 0, 128, 64>(ctx, io);
    if (rounding == TC_ROUND_TRUNC) return run_fdwt<int32_t, 0, TC_ROUND_TRUNC, 128, 64>(ctx, io);
    return run_fdwt<int32_t, 0, TC_ROUND_FLOOR, 128, 64>(ctx, io);
}

cudaError_t launch_idwt_last_color(tc_ctx *ctx, const LevelIO &io, int wavelet, int color, int out_type,
                                   int bits, bool)
{
    if (io.w <= 0 || io.h <= 0) return cudaSuccess;
    if (color != TC_COLOR_DC && io.ncomp < 3) color = TC_COLOR_DC;
    if (wavelet) {
        if (color == TC_COLOR_ICT || color == TC_COLOR_RCT)
            return run_last<float, 1, 0, TC_COLOR_ICT>(ctx, io, out_type, bits);
        return run_last<float, 1, 0, TC_COLOR_DC>(ctx, io, out_type, bits);
    }
    if (color == TC_COLOR_RCT || color == TC_COLOR_ICT)
        return run_last<int32_t, 0, TC_ROUND_FLOOR, TC_COLOR_RCT>(ctx, io, out_type, bits);
    return run_last<int32_t, 0, TC_ROUND_FLOOR, TC_COLOR_DC>(ctx, io, out_type, bits);
}

}  // namespace tc
