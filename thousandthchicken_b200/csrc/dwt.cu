// dwt.cu -- forward 5/3 (int32) and 9/7 (fp32) lifting DWT levels for
// sm_100a (the encoder's and the tc_dwt_forward* entry points; the reverse
// levels are in dwt_rev.cu).
//
// Replaces the reference's forward kernels (dwt_f53.cl, dwt_f97.cl over
// dwt_transform_buffer.cl / dwt_io.cl):
//   * one launch per level; each CTA owns a TX x TY output tile and stages
//     the tile plus a halo of H samples (2 for 5/3, 4 for 9/7) in shared
//     memory with whole-sample symmetric extension (full periodic
//     reflection, ISO F.3.7, instead of the single reflection of
//     dwt_io.cl:7-38, defect D14);
//   * rows are stored split into even/odd halves so every lifting step is a
//     unit-stride, bank-conflict-free sweep; the store deinterleaves the
//     tile straight into the Mallat subbands;
//   * 5/3 uses floor (ISO) or truncating (reference, defect D13) rounding;
//     9/7 uses fp32 with the scaling factors applied as floats (defects
//     D10-D12 fixed).
#include <cuda_runtime.h>

#include "dwt_common.cuh"
#include "tc_internal.cuh"

namespace tc {
namespace {

using namespace dwt;

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

template <typename T, int WAVELET, int RND, int TX, int TY>
cudaError_t run_fdwt(tc_ctx *ctx, const LevelIO &io)
{
    dim3 grid((io.w + TX - 1) / TX, (io.h + TY - 1) / TY, io.ncomp);
    fdwt_level_kernel<T, WAVELET, RND, TX, TY><<<grid, 256, 0, ctx->stream>>>(io);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_fdwt_level(tc_ctx *ctx, const LevelIO &io, int wavelet, int rounding)
{
    if (io.w <= 0 || io.h <= 0) return cudaSuccess;
    if (wavelet) return run_fdwt<float, 1, 0, 128, 64>(ctx, io);
    if (rounding == TC_ROUND_TRUNC) return run_fdwt<int32_t, 0, TC_ROUND_TRUNC, 128, 64>(ctx, io);
    return run_fdwt<int32_t, 0, TC_ROUND_FLOOR, 128, 64>(ctx, io);
}

}  // namespace tc
