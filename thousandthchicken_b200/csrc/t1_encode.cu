// t1_encode.cu -- Tier-1 EBCOT/MQ code-block encoder for sm_100a.
//
// The reference has no Tier-1 encoder; this is the GPU half of the forward
// pipeline (forward colour transform and DWT in color.cu / dwt.cu).  It
// produces, block for block, the same codeword as the project's host encoder
// (t1_encode_block in j2k_host.cpp): all coding passes, or the first
// max_passes of them, MQ termination by the FLUSH procedure of ISO C.2.9.
//
//   * one warp per code-block, CTAs of kEncWarps blocks; at every bit-plane
//     the lanes rebuild the plane's bits per column from the input (float
//     quantised with the band's step, or int32), read coalesced and cached,
//     so a block's state is 5.7 KB of shared memory;
//   * the coding state is the decoder's flag-word layout (t1_common.cuh):
//     at every stripe the lanes find the candidate columns of the pass with
//     __ballot_sync and the serial loop visits only those, in scan order;
//   * the MQ encoder (ISO C.2) keeps A, C, CT and the last output byte in
//     registers, replicated across the lanes; lane 0 writes the bytes once
//     they can no longer take a carry.
#include <cuda_runtime.h>

#include <cmath>

#include "t1_common.cuh"
#include "tc_internal.cuh"

namespace tc {
namespace {

constexpr int kEncWarps = 8;

// A block's coding state: 5.7 KB, so that 32 warps fit an SM.  The
// magnitudes are not kept: at every bit-plane the lanes rebuild that
// plane's bits per column from the (cached) input.
struct EncState {
    uint32_t F[kMaxStripes * 64];       // flag word per stripe column
    unsigned long long sgn[kSgnCols];   // sign of the significant samples per column
    unsigned long long neg[64];         // sign of every sample per column (bit y)
    unsigned long long bits[64];        // the current bit-plane per column (bit y)
    uint32_t ctx[20];                   // packed probability state per context
    uint8_t mrow[64], mctx[64];         // refinement pass: rows and context codes per column
};

// Magnitude of sample (x, y) of block d: the int32 input, or the float input
// quantised floor(|v| / step) (ISO E.2 deadzone).
__device__ __forceinline__ uint32_t magnitude(const tc_t1_enc_desc &d, const void *in, int x, int y)
{
    const size_t i = d.in_off + (size_t)y * d.in_pitch + x;
    if (d.flags & TC_CBLK_IRREVERSIBLE) return (uint32_t)floorf(fabsf(__ldg(static_cast<const float *>(in) + i)) * d.inv_step);
    const int32_t v = __ldg(static_cast<const int32_t *>(in) + i);
    return (uint32_t)(v < 0 ? -(int64_t)v : v);
}

// MQ encoder (ISO C.2.1-C.2.9).  A is 16 bits wide as in the standard; each
// context word is the decoder's packed state (Qe << 16 | NMPS << 1 |
// NLPS << 7 | SWITCH << 13 | MPS).  The last byte emitted (B of the
// standard) stays in a register until the next one is emitted, since a
// carry can still increment it; bytes before it are final.
struct MQEnc {
    uint8_t *out;
    uint32_t cap, n;   // n: bytes emitted so far (B is byte n - 1; n == 0: B is the byte before the codeword)
    uint32_t a, c, b;
    int ct;
    bool writer, overflow;

    __device__ __forceinline__ void init(uint8_t *o, uint32_t capacity, bool w)
    {
        out = o;
        cap = capacity;
        n = 0;
        a = 0x8000u;
        c = 0;
        b = 0;
        ct = 12;
        writer = w;
        overflow = false;
    }
    __device__ __forceinline__ void put(uint32_t v)
    {
        if (n >= 1) {
            if (n - 1 < cap) {
                if (writer) out[n - 1] = (uint8_t)b;
            } else {
                overflow = true;
            }
        }
        n++;
        b = v & 0xFFu;
    }
    __device__ __forceinline__ void byteout()
    {
        if (b == 0xFFu) {
            put(c >> 20);
            c &= 0xFFFFFu;
            ct = 7;
        } else if (c < 0x8000000u) {
            put(c >> 19);
            c &= 0x7FFFFu;
            ct = 8;
        } else {
            b++;
            if (b == 0xFFu) {
                c &= 0x7FFFFFFu;
                put(c >> 20);
                c &= 0xFFFFFu;
                ct = 7;
            } else {
                put(c >> 19);
                c &= 0x7FFFFu;
                ct = 8;
            }
        }
    }
    __device__ __forceinline__ void renorm()
    {
        do {
            a <<= 1;
            c <<= 1;
            if (--ct == 0) byteout();
        } while ((a & 0x8000u) == 0u);
    }
    __device__ __forceinline__ void encode(uint32_t *ctx, const uint32_t *tbl, int cx, uint32_t d)
    {
        const uint32_t w = ctx[cx];
        const uint32_t qe = w >> 16, mps = w & 1u;
        a -= qe;
        if (d == mps) {
            if ((a & 0x8000u) == 0u) {
                if (a < qe) a = qe;
                else c += qe;
                ctx[cx] = tbl[(w >> 1) & 63] | mps;
                renorm();
            } else {
                c += qe;
            }
        } else {
            if (a < qe) c += qe;
            else a = qe;
            ctx[cx] = tbl[(w >> 7) & 63] | (mps ^ ((w >> 13) & 1u));
            renorm();
        }
    }
    // FLUSH (ISO C.2.9); returns the codeword length (a final 0xFF dropped).
    __device__ __forceinline__ uint32_t flush()
    {
        const uint32_t tempc = c + a;
        c |= 0xFFFFu;
        if (c >= tempc) c -= 0x8000u;
        c <<= ct;
        byteout();
        c <<= ct;
        byteout();
        const uint32_t len = b == 0xFFu ? n - 1 : n;
        if (n >= 1 && n - 1 < len) {  // the last byte is part of the codeword
            if (n - 1 < cap) {
                if (writer) out[n - 1] = (uint8_t)b;
            } else {
                overflow = true;
            }
        }
        return len;
    }
};

// The first `limit` coding passes of a block whose state S holds the signs
// and a cleared coding state (the lanes in lock-step; limit is the same in
// every lane, so the early exits are uniform).
__device__ void encode_block(EncState &S, const Tables &T, MQEnc &mq, const tc_t1_enc_desc &d, const void *in,
                             int numbps, int limit, int lane)
{
    const int w = d.w, h = d.h, orient = d.orient;
    uint32_t *ctx = S.ctx;
    const uint32_t *tbl = T.mq;
    const uint8_t *zc = T.zc[orient];
    uint32_t *F = S.F;
    const int nstripes = (h + 3) >> 2;
    constexpr int G = 32, CPL = 2;
    const unsigned gmask = 0xffffffffu;
    auto bit = [&](int y, int c, int) -> uint32_t { return (uint32_t)(S.bits[c] >> y) & 1u; };
    auto sign_bit = [&](int y, int c) -> uint32_t { return (uint32_t)(S.neg[c] >> y) & 1u; };

    int done = 0;  // coding passes emitted
    for (int p = numbps - 1; p >= 0 && done < limit; --p) {
        // this bit-plane's bits, the lanes' columns
#pragma unroll
        for (int j = 0; j < CPL; j++) {
            const int c = lane + G * j;
            unsigned long long m = 0;
            if (c < w)
                for (int y = 0; y < h; y++) m |= (unsigned long long)((magnitude(d, in, c, y) >> p) & 1u) << y;
            S.bits[c] = m;
        }
        __syncwarp();
        if (p != numbps - 1) {
            // ---- significance propagation pass (ISO D.3.1) ----
            for (int s = 0; s < nstripes; s++) {
                const int rows = min(4, h - 4 * s);
                __syncwarp();
                bool any[CPL];
#pragma unroll
                for (int j = 0; j < CPL; j++) {
                    const int c = lane + G * j;
                    bool a = false;
                    if (c < w) {
                        const uint32_t f = F[s * 64 + c];
                        for (int k = 0; k < rows; k++) a |= !(f & self_bit(k)) && ((f >> (3 * k)) & 0x1EFu);
                    }
                    any[j] = a;
                }
                unsigned long long cand = group_ballot<G>(any, gmask, 0);
                while (cand) {
                    const int c = __ffsll((long long)cand) - 1;
                    cand &= cand - 1;
                    uint32_t f = F[s * 64 + c];
                    const uint32_t f0 = f;
                    for (int k = 0; k < rows; k++) {
                        if (f & self_bit(k)) continue;
                        const uint32_t n9 = (f >> (3 * k)) & 0x1FFu;
                        if (!(n9 & 0x1EFu)) continue;
                        f |= pi_bit(k);
                        const int y = 4 * s + k;
                        const uint32_t b = bit(y, c, p);
                        mq.encode(ctx, tbl, zc[n9], b);
                        if (b) {
                            const uint32_t si = T.sc[sign_index(S.sgn, n9, c, y)];
                            const uint32_t neg = sign_bit(y, c);
                            mq.encode(ctx, tbl, si & 15, neg ^ (si >> 4));
                            f |= self_bit(k);
                            mark_significant(F, S.sgn, s, k, c, w, nstripes, neg);
                            if (c + 1 < w) cand |= 1ull << (c + 1);  // the next column gained a neighbour
                        }
                    }
                    if (f != f0) F[s * 64 + c] = f;
                }
            }
            if (++done >= limit) break;

            // ---- magnitude refinement pass (ISO D.3.3) ----
            for (int s = 0; s < nstripes; s++) {
                const int rows = min(4, h - 4 * s);
                __syncwarp();
                bool any[CPL];
#pragma unroll
                for (int j = 0; j < CPL; j++) {
                    const int c = lane + G * j;
                    uint32_t rr = 0, codes = 0;
                    if (c < w) {
                        const uint32_t f = F[s * 64 + c];
                        for (int k = 0; k < rows; k++) {
                            if ((f & self_bit(k)) && !(f & pi_bit(k))) {
                                rr |= 1u << k;
                                const uint32_t code = (f & ref_bit(k)) ? 2u : (((f >> (3 * k)) & 0x1EFu) ? 1u : 0u);
                                codes |= code << (2 * k);
                            }
                        }
                        S.mrow[c] = (uint8_t)rr;
                        S.mctx[c] = (uint8_t)codes;
                        if (rr) F[s * 64 + c] = f | (rr << 22);
                    }
                    any[j] = rr != 0;
                }
                unsigned long long cand = group_ballot<G>(any, gmask, 0);
                __syncwarp();
                while (cand) {
                    const int c = __ffsll((long long)cand) - 1;
                    cand &= cand - 1;
                    uint32_t rr = S.mrow[c];
                    const uint32_t codes = S.mctx[c];
                    while (rr) {
                        const int k = __ffs(rr) - 1;
                        rr &= rr - 1;
                        mq.encode(ctx, tbl, 14 + ((codes >> (2 * k)) & 3u), bit(4 * s + k, c, p));
                    }
                }
            }
            if (++done >= limit) break;
        }

        // ---- cleanup pass (ISO D.3.4) ----
        for (int s = 0; s < nstripes; s++) {
            const int rows = min(4, h - 4 * s);
            const uint32_t rmask = (1u << rows) - 1u;
            __syncwarp();
            bool any[CPL];
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                const int c = lane + G * j;
                bool a = false;
                if (c < w) {
                    const uint32_t f = F[s * 64 + c];
                    uint32_t done = (f >> 18) & 0xFu;  // pi
#pragma unroll
                    for (int k = 0; k < 4; k++) done |= ((f >> (3 * k + 4)) & 1u) << k;
                    a = (~done & rmask) != 0u;
                }
                any[j] = a;
            }
            unsigned long long cand = group_ballot<G>(any, gmask, 0);
            while (cand) {
                const int c = __ffsll((long long)cand) - 1;
                cand &= cand - 1;
                uint32_t f = F[s * 64 + c];
                const uint32_t f0 = f;
                int k = 0;
                if (rows == 4 && (f & kSigMask) == 0u) {
                    // run-length mode: four rows with an all-zero neighbourhood
                    const uint32_t four = (uint32_t)(S.bits[c] >> (4 * s)) & 0xFu;
                    const int r = four ? __ffs(four) - 1 : -1;
                    if (r < 0) {
                        mq.encode(ctx, tbl, 18, 0u);
                        continue;
                    }
                    mq.encode(ctx, tbl, 18, 1u);
                    mq.encode(ctx, tbl, 17, (uint32_t)(r >> 1));
                    mq.encode(ctx, tbl, 17, (uint32_t)(r & 1));
                    const int y = 4 * s + r;
                    const uint32_t si = T.sc[sign_index(S.sgn, (f >> (3 * r)) & 0x1FFu, c, y)];
                    const uint32_t neg = sign_bit(y, c);
                    mq.encode(ctx, tbl, si & 15, neg ^ (si >> 4));
                    f |= self_bit(r);
                    mark_significant(F, S.sgn, s, r, c, w, nstripes, neg);
                    k = r + 1;
                }
                for (; k < rows; k++) {
                    if (f & (self_bit(k) | pi_bit(k))) continue;
                    const uint32_t n9 = (f >> (3 * k)) & 0x1FFu;
                    const int y = 4 * s + k;
                    const uint32_t b = bit(y, c, p);
                    mq.encode(ctx, tbl, zc[n9], b);
                    if (b) {
                        const uint32_t si = T.sc[sign_index(S.sgn, n9, c, y)];
                        const uint32_t neg = sign_bit(y, c);
                        mq.encode(ctx, tbl, si & 15, neg ^ (si >> 4));
                        f |= self_bit(k);
                        mark_significant(F, S.sgn, s, k, c, w, nstripes, neg);
                    }
                }
                if (f != f0) F[s * 64 + c] = f;
            }
        }
        ++done;
        __syncwarp();
        for (int i = lane; i < nstripes * 64; i += G) F[i] &= ~0x3C0000u;  // clear pi
        __syncwarp();
    }
}

// One code-block per warp; blocks b = blockIdx.x * kEncWarps + warp.
__global__ void __launch_bounds__(32 * kEncWarps)
    t1_encode_kernel(const tc_t1_enc_desc *__restrict__ desc, int n, const void *__restrict__ in,
                     uint8_t *__restrict__ out, uint32_t cap, tc_t1_enc_result *__restrict__ res)
{
    extern __shared__ __align__(16) unsigned char smem[];
    Tables &T = *reinterpret_cast<Tables *>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    EncState &S = reinterpret_cast<EncState *>(smem + ((sizeof(Tables) + 15) & ~size_t(15)))[warp];
    build_tables(T);
    __syncthreads();
    const int bi = blockIdx.x * kEncWarps + warp;
    if (bi >= n) return;
    const tc_t1_enc_desc d = desc[bi];
    const int w = d.w, h = d.h;
    tc_t1_enc_result r{0u, 0u, 0u, 0u};
    if (w < 1 || w > 64 || h < 1 || h > 64 || d.orient > 3 || d.mb < 1 || d.mb > 31) {
        r.status = 1;
        if (lane == 0) res[bi] = r;
        return;
    }
    // largest magnitude and the signs, rows coalesced across the lanes
    const bool irrev = (d.flags & TC_CBLK_IRREVERSIBLE) != 0;
    uint32_t mx = 0;
    unsigned long long neg0 = 0, neg1 = 0;  // columns lane and lane + 32
    for (int y = 0; y < h; y++) {
        const size_t row = d.in_off + (size_t)y * d.in_pitch;
        for (int j = 0; j < 2; j++) {
            const int x = lane + 32 * j;
            if (x >= w) continue;
            const uint32_t m = magnitude(d, in, x, y);
            const bool ng = irrev ? static_cast<const float *>(in)[row + x] < 0.0f
                                  : static_cast<const int32_t *>(in)[row + x] < 0;
            mx = max(mx, m);
            if (ng && m) (j ? neg1 : neg0) |= 1ull << y;
        }
    }
    S.neg[lane] = neg0;
    S.neg[lane + 32] = neg1;
    for (int i = lane; i < kMaxStripes * 64; i += 32) S.F[i] = 0u;
    for (int i = lane; i < kSgnCols; i += 32) S.sgn[i] = 0ull;
    for (int i = lane; i < 19; i += 32) {
        const int st = i == 0 ? 4 : (i == 17 ? 46 : (i == 18 ? 3 : 0));
        S.ctx[i] = T.mq[st];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    __syncwarp();
    const int numbps = 32 - __clz(mx);
    if (numbps > d.mb) {
        r.status = 2;  // the magnitudes need more bit-planes than the band has
    } else if (numbps > 0) {
        // passes kept: d.max_passes (0 or more than the block has: all)
        const int total = 3 * numbps - 2;
        const int limit = d.max_passes && d.max_passes < total ? (int)d.max_passes : total;
        MQEnc mq;
        mq.init(out + (size_t)bi * cap, cap, lane == 0);
        encode_block(S, T, mq, d, in, numbps, limit, lane);
        r.len = mq.flush();
        r.passes = (uint32_t)limit;
        if (mq.overflow || r.len > cap) {
            r.status = 3;
            r.len = 0;
        }
    }
    r.zero_bitplanes = (uint32_t)(d.mb - min(numbps, (int)d.mb));
    if (lane == 0) res[bi] = r;
}

constexpr size_t kEncSmem = ((sizeof(Tables) + 15) & ~size_t(15)) + kEncWarps * sizeof(EncState);

}  // namespace

cudaError_t launch_t1_encode(tc_ctx *ctx, const tc_t1_enc_desc *d_desc, int n, const void *d_in, uint8_t *d_out,
                             uint32_t cap, tc_t1_enc_result *d_res)
{
    if (n <= 0) return cudaSuccess;
    static DeviceFlags attr;
    if (cudaError_t e = set_smem_once(attr, ctx->device, t1_encode_kernel, kEncSmem)) return e;
    t1_encode_kernel<<<(n + kEncWarps - 1) / kEncWarps, 32 * kEncWarps, kEncSmem, ctx->stream>>>(d_desc, n, d_in, d_out,
                                                                                               cap, d_res);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace tc

namespace tc {
namespace {

// Packs the codewords: block k's len[k] bytes from src + k * cap to
// dst + off[k] (one CTA per block).
__global__ void gather_codewords_kernel(const uint8_t *__restrict__ src, uint32_t cap,
                                        const tc_t1_enc_result *__restrict__ res, const uint64_t *__restrict__ off,
                                        int n, uint8_t *__restrict__ dst)
{
    const int k = blockIdx.x;
    if (k >= n) return;
    const uint32_t len = res[k].len;
    const uint8_t *s = src + (size_t)k * cap;
    uint8_t *d = dst + off[k];
    for (uint32_t i = threadIdx.x; i < len && i < cap; i += blockDim.x) d[i] = s[i];
}

}  // namespace

cudaError_t launch_gather_codewords(tc_ctx *ctx, const uint8_t *src, uint32_t cap, const tc_t1_enc_result *res,
                                    const uint64_t *off, int n, uint8_t *dst)
{
    if (n <= 0) return cudaSuccess;
    gather_codewords_kernel<<<n, 128, 0, ctx->stream>>>(src, cap, res, off, n, dst);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace tc
