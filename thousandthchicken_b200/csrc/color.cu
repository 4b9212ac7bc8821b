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

template <typename OT>
__device__ __forceinline__ OT clamped(int v, int lo, int hi)
{
    return (OT)(v < lo ? lo : (v > hi ? hi : v));
}

// Four consecutive samples of a row: one 16-byte (or 8/4-byte) access when
// the row is aligned for it, else four scalar accesses; `n` of them valid.
template <typename T>
__device__ __forceinline__ void load4(const T *p, bool vec, int n, T (&v)[4])
{
    if (vec && n == 4) {
        if constexpr (sizeof(T) == 4) {
            const int4 q = *reinterpret_cast<const int4 *>(p);
            if constexpr (std::is_integral<T>::value) {
                v[0] = (T)q.x, v[1] = (T)q.y, v[2] = (T)q.z, v[3] = (T)q.w;
            } else {
                v[0] = __int_as_float(q.x), v[1] = __int_as_float(q.y), v[2] = __int_as_float(q.z),
                v[3] = __int_as_float(q.w);
            }
        } else if constexpr (sizeof(T) == 2) {
            const uint2 q = *reinterpret_cast<const uint2 *>(p);
            v[0] = (T)(q.x & 0xFFFFu), v[1] = (T)(q.x >> 16), v[2] = (T)(q.y & 0xFFFFu), v[3] = (T)(q.y >> 16);
        } else {
            const uint32_t q = *reinterpret_cast<const uint32_t *>(p);
            v[0] = (T)(q & 0xFF), v[1] = (T)((q >> 8) & 0xFF), v[2] = (T)((q >> 16) & 0xFF), v[3] = (T)(q >> 24);
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < 4; j++) v[j] = j < n ? p[j] : T(0);
}

template <typename T>
__device__ __forceinline__ void store4(T *p, bool vec, int n, const T (&v)[4])
{
    if (vec && n == 4) {
        if constexpr (sizeof(T) == 4) {
            int4 q;
            if constexpr (std::is_integral<T>::value) q = make_int4(v[0], v[1], v[2], v[3]);
            else q = make_int4(__float_as_int(v[0]), __float_as_int(v[1]), __float_as_int(v[2]), __float_as_int(v[3]));
            *reinterpret_cast<int4 *>(p) = q;
        } else if constexpr (sizeof(T) == 2) {
            *reinterpret_cast<uint2 *>(p) = make_uint2((uint32_t)(uint16_t)v[0] | ((uint32_t)(uint16_t)v[1] << 16),
                                                       (uint32_t)(uint16_t)v[2] | ((uint32_t)(uint16_t)v[3] << 16));
        } else {
            *reinterpret_cast<uint32_t *>(p) = (uint32_t)(uint8_t)v[0] | ((uint32_t)(uint8_t)v[1] << 8) |
                                               ((uint32_t)(uint8_t)v[2] << 16) | ((uint32_t)(uint8_t)v[3] << 24);
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (j < n) p[j] = v[j];
}

// Launch shape shared by the colour kernels: a thread covers four
// consecutive samples of a row; blockIdx.y strides over rows.
constexpr int kColThreads = 256;

inline dim3 color_grid(int w, int h)
{
    const int gx = (w + 4 * kColThreads - 1) / (4 * kColThreads);
    int gy = (148 * 16 + gx - 1) / gx;
    if (gy > h) gy = h;
    return dim3(gx, gy < 1 ? 1 : gy);
}

// Inverse: IT = int32_t or float input planes; OT = output sample type.
// vin / vout: every input / output row is aligned for 4-sample accesses.
template <typename IT, typename OT, int KIND, int NC>
__global__ void __launch_bounds__(kColThreads) color_inverse_kernel(Planes P, int in_pitch, int out_pitch, int w,
                                                                    int h, int bits, bool vin, bool vout)
{
    const int x0 = 4 * (blockIdx.x * kColThreads + threadIdx.x);
    if (x0 >= w) return;
    const int n = min(4, w - x0);
    const OutRange R = out_range(bits);
    for (int y = blockIdx.y; y < h; y += gridDim.y) {
        const size_t ii = (size_t)y * in_pitch + x0, oi = (size_t)y * out_pitch + x0;
        IT a[NC][4];
#pragma unroll
        for (int c = 0; c < NC; c++) load4<IT>(static_cast<const IT *>(P.in[c]) + ii, vin, n, a[c]);
        OT o[NC][4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int v[NC];
            if constexpr (KIND == TC_COLOR_RCT && NC >= 3) {
                // tcr_kernel, preprocess_rct_inverse.cl:18-36
                const int Y = (int)a[0][j], U = (int)a[1][j], V = (int)a[2][j];
                const int G = Y - ((U + V) >> 2);
                v[0] = V + G;
                v[1] = G;
                v[2] = U + G;
            } else if constexpr (KIND == TC_COLOR_ICT && NC >= 3) {
                // ISO G.2 inverse ICT (tci_kernel's constants are defect D9)
                const float Y = (float)a[0][j], Cb = (float)a[1][j], Cr = (float)a[2][j];
                v[0] = __float2int_rn(fmaf(1.402f, Cr, Y));
                v[1] = __float2int_rn(Y - 0.34413f * Cb - 0.71414f * Cr);
                v[2] = __float2int_rn(fmaf(1.772f, Cb, Y));
            }
            constexpr int c0 = (KIND != TC_COLOR_DC && NC >= 3) ? 3 : 0;
#pragma unroll
            for (int c = c0; c < NC; c++) {
                if constexpr (std::is_integral<IT>::value) v[c] = (int)a[c][j];
                else v[c] = __float2int_rn((float)a[c][j]);
            }
#pragma unroll
            for (int c = 0; c < NC; c++) o[c][j] = clamped<OT>(v[c] + R.dc, R.lo, R.hi);
        }
#pragma unroll
        for (int c = 0; c < NC; c++) store4<OT>(static_cast<OT *>(P.out[c]) + oi, vout, n, o[c]);
    }
}

// Forward: unsigned samples -> DC shift + RCT (int32 out) / ICT (float out)
// / DC only (int32 or float out).
template <typename IT, typename OT, int KIND, int NC>
__global__ void __launch_bounds__(kColThreads) color_forward_kernel(Planes P, int in_pitch, int out_pitch, int w,
                                                                    int h, int bits, bool vin, bool vout)
{
    const int x0 = 4 * (blockIdx.x * kColThreads + threadIdx.x);
    if (x0 >= w) return;
    const int n = min(4, w - x0);
    const int dc = out_range(bits).dc;
    const bool sgn = bits & TC_SIGNED;
    for (int y = blockIdx.y; y < h; y += gridDim.y) {
        const size_t ii = (size_t)y * in_pitch + x0, oi = (size_t)y * out_pitch + x0;
        IT a[NC][4];
#pragma unroll
        for (int c = 0; c < NC; c++) load4<IT>(static_cast<const IT *>(P.in[c]) + ii, vin, n, a[c]);
        OT o[NC][4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int s_[NC];
#pragma unroll
            for (int c = 0; c < NC; c++) {
                int v = (int)a[c][j];
                // signed samples arrive in two's complement
                if constexpr (sizeof(IT) == 1) v = sgn ? (int)(int8_t)a[c][j] : v;
                if constexpr (sizeof(IT) == 2) v = sgn ? (int)(int16_t)a[c][j] : v;
                s_[c] = v - dc;
            }
            int c0 = 0;
            if constexpr (KIND == TC_COLOR_RCT && NC >= 3) {
                // rct_kernel, preprocess_rct.cl:18-31
                o[0][j] = (OT)((s_[0] + 2 * s_[1] + s_[2]) >> 2);
                o[1][j] = (OT)(s_[2] - s_[1]);
                o[2][j] = (OT)(s_[0] - s_[1]);
                c0 = 3;
            } else if constexpr (KIND == TC_COLOR_ICT && NC >= 3) {
                // ict_kernel, preprocess_ict.cl:20-37 (kept in float, no rounding)
                const float R = (float)s_[0], G = (float)s_[1], B = (float)s_[2];
                const float Y = 0.299f * R + 0.587f * G + 0.114f * B;
                const float Cb = -0.16875f * R - 0.33126f * G + 0.5f * B;
                const float Cr = 0.5f * R - 0.41869f * G - 0.08131f * B;
                if constexpr (std::is_integral<OT>::value) {
                    // integer output rounds to nearest even like ict_kernel's convert_int_sat_rte
                    o[0][j] = (OT)__float2int_rn(Y);
                    o[1][j] = (OT)__float2int_rn(Cb);
                    o[2][j] = (OT)__float2int_rn(Cr);
                } else {
                    o[0][j] = Y;
                    o[1][j] = Cb;
                    o[2][j] = Cr;
                }
                c0 = 3;
            }
#pragma unroll
            for (int c = 0; c < NC; c++)
                if (c >= c0) o[c][j] = (OT)s_[c];
        }
#pragma unroll
        for (int c = 0; c < NC; c++) store4<OT>(static_cast<OT *>(P.out[c]) + oi, vout, n, o[c]);
    }
}

// Whether every row of every plane starts aligned for 4-sample accesses.
bool rows_aligned(const void *const *planes, int ncomp, int pitch, size_t elem)
{
    const size_t a = 4 * elem;
    if (((size_t)pitch * elem) % a) return false;
    for (int c = 0; c < ncomp; c++)
        if (reinterpret_cast<uintptr_t>(planes[c]) % a) return false;
    return true;
}

template <typename IT, typename OT, int KIND>
cudaError_t inv_launch(tc_ctx *ctx, int ncomp, const Planes &P, int ip, int op, int w, int h, int bits, bool vi,
                       bool vo)
{
    const dim3 g = color_grid(w, h);
    switch (ncomp) {
    case 1: color_inverse_kernel<IT, OT, KIND, 1><<<g, kColThreads, 0, ctx->stream>>>(P, ip, op, w, h, bits, vi, vo); break;
    case 2: color_inverse_kernel<IT, OT, KIND, 2><<<g, kColThreads, 0, ctx->stream>>>(P, ip, op, w, h, bits, vi, vo); break;
    case 3: color_inverse_kernel<IT, OT, KIND, 3><<<g, kColThreads, 0, ctx->stream>>>(P, ip, op, w, h, bits, vi, vo); break;
    default: color_inverse_kernel<IT, OT, KIND, 4><<<g, kColThreads, 0, ctx->stream>>>(P, ip, op, w, h, bits, vi, vo); break;
    }
    ctx->launches++;
    return cudaGetLastError();
}

template <typename IT, typename OT>
cudaError_t inv_dispatch(tc_ctx *ctx, int kind, const Planes &P, int ncomp, int ip, int op, int w, int h,
                         int bits)
{
    const bool vi = rows_aligned(P.in, ncomp, ip, sizeof(IT)), vo = rows_aligned(P.out, ncomp, op, sizeof(OT));
    if (kind == TC_COLOR_RCT) return inv_launch<IT, OT, TC_COLOR_RCT>(ctx, ncomp, P, ip, op, w, h, bits, vi, vo);
    if (kind == TC_COLOR_ICT) return inv_launch<IT, OT, TC_COLOR_ICT>(ctx, ncomp, P, ip, op, w, h, bits, vi, vo);
    return inv_launch<IT, OT, TC_COLOR_DC>(ctx, ncomp, P, ip, op, w, h, bits, vi, vo);
}

template <typename IT, typename OT, int KIND>
cudaError_t fwd_launch(tc_ctx *ctx, int ncomp, const Planes &P, int ip, int op, int w, int h, int bits, bool vi,
                       bool vo)
{
    const dim3 g = color_grid(w, h);
    switch (ncomp) {
    case 1: color_forward_kernel<IT, OT, KIND, 1><<<g, kColThreads, 0, ctx->stream>>>(P, ip, op, w, h, bits, vi, vo); break;
    case 2: color_forward_kernel<IT, OT, KIND, 2><<<g, kColThreads, 0, ctx->stream>>>(P, ip, op, w, h, bits, vi, vo); break;
    case 3: color_forward_kernel<IT, OT, KIND, 3><<<g, kColThreads, 0, ctx->stream>>>(P, ip, op, w, h, bits, vi, vo); break;
    default: color_forward_kernel<IT, OT, KIND, 4><<<g, kColThreads, 0, ctx->stream>>>(P, ip, op, w, h, bits, vi, vo); break;
    }
    ctx->launches++;
    return cudaGetLastError();
}

template <typename IT, typename OT>
cudaError_t fwd_dispatch(tc_ctx *ctx, int kind, const Planes &P, int ncomp, int ip, int op, int w, int h,
                         int bits)
{
    const bool vi = rows_aligned(P.in, ncomp, ip, sizeof(IT)), vo = rows_aligned(P.out, ncomp, op, sizeof(OT));
    if (kind == TC_COLOR_RCT) return fwd_launch<IT, OT, TC_COLOR_RCT>(ctx, ncomp, P, ip, op, w, h, bits, vi, vo);
    if (kind == TC_COLOR_ICT) return fwd_launch<IT, OT, TC_COLOR_ICT>(ctx, ncomp, P, ip, op, w, h, bits, vi, vo);
    return fwd_launch<IT, OT, TC_COLOR_DC>(ctx, ncomp, P, ip, op, w, h, bits, vi, vo);
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
