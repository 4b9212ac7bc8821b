// color.cu -- standalone component transforms and DC level shift.
//
// The Preprocessor stage of the reference (Preprocessor.cpp:44-306, kernels
// preprocess_rct*.cl, preprocess_ict*.cl, preprocess_dc_level_shift*.cl) as
// plane-wise, vectorisable element kernels.  The decode pipeline fuses the
// inverse path into the last DWT level; these kernels serve the standalone
// Preprocessor API and the forward (encoder-side) path.
#include <cuda_runtime.h>

#include <type_traits>

#include "tc_internal.cuh"

namespace tc {
namespace {

struct Planes {
    const void *in[4];
    void *out[4];
};

template <typename T>
__device__ __forceinline__ float ldf(const void *p, size_t i)
{
    return (float)static_cast<const T *>(p)[i];
}

template <typename IT>
__device__ __forceinline__ IT ld(const void *p, size_t i)
{
    return static_cast<const IT *>(p)[i];
}

template <typename OT>
__device__ __forceinline__ void st_clamped(void *p, size_t i, int v, int mx)
{
    static_cast<OT *>(p)[i] = (OT)(v < 0 ? 0 : (v > mx ? mx : v));
}

// Inverse: IT = int32_t or float input planes; OT = output sample type.
template <typename IT, typename OT, int KIND>
__global__ void color_inverse_kernel(Planes P, int ncomp, int in_pitch, int out_pitch, int w, int h,
                                     int bits)
{
    const size_t n = (size_t)w * h;
    const int dc = 1 << (bits - 1), mx = (1 << bits) - 1;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(q / w), x = (int)(q % w);
        const size_t ii = (size_t)y * in_pitch + x, oi = (size_t)y * out_pitch + x;
        int v[4];
        for (int c = 0; c < ncomp; c++) {
            if constexpr (std::is_integral<IT>::value) v[c] = (int)ld<IT>(P.in[c], ii);
            else v[c] = __float2int_rn((float)ld<IT>(P.in[c], ii));
        }
        if constexpr (KIND == TC_COLOR_RCT) {
            // tcr_kernel, preprocess_rct_inverse.cl:18-36
            const int Y = (int)ld<IT>(P.in[0], ii), U = (int)ld<IT>(P.in[1], ii), V = (int)ld<IT>(P.in[2], ii);
            const int G = Y - ((U + V) >> 2);
            v[0] = V + G;
            v[1] = G;
            v[2] = U + G;
        } else if constexpr (KIND == TC_COLOR_ICT) {
            // ISO G.2 inverse ICT (tci_kernel's constants are defect D9)
            const float Y = (float)ld<IT>(P.in[0], ii), Cb = (float)ld<IT>(P.in[1], ii),
                        Cr = (float)ld<IT>(P.in[2], ii);
            v[0] = __float2int_rn(fmaf(1.402f, Cr, Y));
            v[1] = __float2int_rn(Y - 0.34413f * Cb - 0.71414f * Cr);
            v[2] = __float2int_rn(fmaf(1.772f, Cb, Y));
        }
        for (int c = 0; c < ncomp; c++) st_clamped<OT>(P.out[c], oi, v[c] + dc, mx);
    }
}

// Forward: unsigned samples -> DC shift + RCT (int32 out) / ICT (float out)
// / DC only (int32 or float out).
template <typename IT, typename OT, int KIND>
__global__ void color_forward_kernel(Planes P, int ncomp, int in_pitch, int out_pitch, int w, int h,
                                     int bits)
{
    const size_t n = (size_t)w * h;
    const int dc = 1 << (bits - 1);
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(q / w), x = (int)(q % w);
        const size_t ii = (size_t)y * in_pitch + x, oi = (size_t)y * out_pitch + x;
        int s[4];
        for (int c = 0; c < ncomp; c++) s[c] = (int)ld<IT>(P.in[c], ii) - dc;
        int c0 = 0;
        if constexpr (KIND == TC_COLOR_RCT) {
            // rct_kernel, preprocess_rct.cl:18-31
            static_cast<OT *>(P.out[0])[oi] = (OT)((s[0] + 2 * s[1] + s[2]) >> 2);
            static_cast<OT *>(P.out[1])[oi] = (OT)(s[2] - s[1]);
            static_cast<OT *>(P.out[2])[oi] = (OT)(s[0] - s[1]);
            c0 = 3;
        } else if constexpr (KIND == TC_COLOR_ICT) {
            // ict_kernel, preprocess_ict.cl:20-37 (kept in float, no rounding)
            const float R = (float)s[0], G = (float)s[1], B = (float)s[2];
            const float Y = 0.299f * R + 0.587f * G + 0.114f * B;
            const float Cb = -0.16875f * R - 0.33126f * G + 0.5f * B;
            const float Cr = 0.5f * R - 0.41869f * G - 0.08131f * B;
            if constexpr (std::is_integral<OT>::value) {
                // integer output rounds to nearest even like ict_kernel's convert_int_sat_rte
                static_cast<OT *>(P.out[0])[oi] = (OT)__float2int_rn(Y);
                static_cast<OT *>(P.out[1])[oi] = (OT)__float2int_rn(Cb);
                static_cast<OT *>(P.out[2])[oi] = (OT)__float2int_rn(Cr);
            } else {
                static_cast<OT *>(P.out[0])[oi] = Y;
                static_cast<OT *>(P.out[1])[oi] = Cb;
                static_cast<OT *>(P.out[2])[oi] = Cr;
            }
            c0 = 3;
        }
        for (int c = c0; c < ncomp; c++) static_cast<OT *>(P.out[c])[oi] = (OT)s[c];
    }
}

int grid_for(size_t n)
{
    const size_t b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

template <typename IT, typename OT>
cudaError_t inv_dispatch(tc_ctx *ctx, int kind, const Planes &P, int ncomp, int ip, int op, int w, int h,
                         int bits)
{
    const int g = grid_for((size_t)w * h);
    if (kind == TC_COLOR_RCT)
        color_inverse_kernel<IT, OT, TC_COLOR_RCT><<<g, 256, 0, ctx->stream>>>(P, ncomp, ip, op, w, h, bits);
    else if (kind == TC_COLOR_ICT)
        color_inverse_kernel<IT, OT, TC_COLOR_ICT><<<g, 256, 0, ctx->stream>>>(P, ncomp, ip, op, w, h, bits);
    else
        color_inverse_kernel<IT, OT, TC_COLOR_DC><<<g, 256, 0, ctx->stream>>>(P, ncomp, ip, op, w, h, bits);
    ctx->launches++;
    return cudaGetLastError();
}

template <typename IT, typename OT>
cudaError_t fwd_dispatch(tc_ctx *ctx, int kind, const Planes &P, int ncomp, int ip, int op, int w, int h,
                         int bits)
{
    const int g = grid_for((size_t)w * h);
    if (kind == TC_COLOR_RCT)
        color_forward_kernel<IT, OT, TC_COLOR_RCT><<<g, 256, 0, ctx->stream>>>(P, ncomp, ip, op, w, h, bits);
    else if (kind == TC_COLOR_ICT)
        color_forward_kernel<IT, OT, TC_COLOR_ICT><<<g, 256, 0, ctx->stream>>>(P, ncomp, ip, op, w, h, bits);
    else
        color_forward_kernel<IT, OT, TC_COLOR_DC><<<g, 256, 0, ctx->stream>>>(P, ncomp, ip, op, w, h, bits);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_color_inverse(tc_ctx *ctx, int kind, int ncomp, void *const *in, int in_type, int in_pitch,
                                 void *const *out, int out_type, int out_pitch, int w, int h, int bits)
{
    Planes P{};
    for (int c = 0; c < ncomp; c++) {
        P.in[c] = in[c];
        P.out[c] = out[c];
    }
    if (in_type == TC_FLOAT32) {
        if (out_type == TC_U8) return inv_dispatch<float, uint8_t>(ctx, kind, P, ncomp, in_pitch, out_pitch, w, h, bits);
        if (out_type == TC_U16) return inv_dispatch<float, uint16_t>(ctx, kind, P, ncomp, in_pitch, out_pitch, w, h, bits);
        return inv_dispatch<float, int32_t>(ctx, kind, P, ncomp, in_pitch, out_pitch, w, h, bits);
    }
    if (out_type == TC_U8) return inv_dispatch<int32_t, uint8_t>(ctx, kind, P, ncomp, in_pitch, out_pitch, w, h, bits);
    if (out_type == TC_U16) return inv_dispatch<int32_t, uint16_t>(ctx, kind, P, ncomp, in_pitch, out_pitch, w, h, bits);
    return inv_dispatch<int32_t, int32_t>(ctx, kind, P, ncomp, in_pitch, out_pitch, w, h, bits);
}

cudaError_t launch_color_forward(tc_ctx *ctx, int kind, int ncomp, const void *const *in, int in_type,
                                 int in_pitch, void *const *out, int out_type, int out_pitch, int w, int h,
                                 int bits)
{
    Planes P{};
    for (int c = 0; c < ncomp; c++) {
        P.in[c] = in[c];
        P.out[c] = out[c];
    }
#define FWD_OUT(IT)                                                                                     \
    (out_type == TC_FLOAT32 ? fwd_dispatch<IT, float>(ctx, kind, P, ncomp, in_pitch, out_pitch, w, h, bits) \
                            : fwd_dispatch<IT, int32_t>(ctx, kind, P, ncomp, in_pitch, out_pitch, w, h, bits))
    if (in_type == TC_U8) return FWD_OUT(uint8_t);
    if (in_type == TC_U16) return FWD_OUT(uint16_t);
    return FWD_OUT(int32_t);
#undef FWD_OUT
}

}  // namespace tc
