// t1_decode.cu -- Tier-1 EBCOT/MQ code-block decoder for sm_100a.
//
// Replaces the reference g_decode kernel (coefficient_coder.cl:778-819) and
// the dequantiser kernels (quantizer_*_inverse.cl) with persistent launches:
//   * one warp per code-block; warps pull block indices from a device work
//     queue (an atomic counter over a longest-first order), so blocks of
//     uneven size and pass count from many tiles and images share a launch;
//   * blocks are split by coded bit-planes (<= 8, <= 16, <= 31) into classes:
//     8-bit magnitudes in shared memory, deeper ones in the block's output
//     words (or as 16- or 32-bit values in shared memory when the launch is
//     small); the classes run as concurrent launches, heaviest first;
//   * the code-block state is one 32-bit flag word per stripe column: the
//     significance of its 3x6 neighbourhood interleaved so that row k's 3x3
//     neighbourhood is (F >> 3k) & 0x1FF, the visited (pi) and refined
//     (sigma') bits of its four rows, and the signs of its six rows (-1..4).
//     A context label is one shift, one mask and one table lookup, a sign
//     context reads the column's word and its two neighbours'; a coefficient
//     that becomes significant updates the words of its neighbours.  (The
//     reference rebuilds a 3x3 window of packed words from global memory at
//     every step, coefficient_coder.cl:271-298.)
//   * the MQ context words carry both successor states whole (Qe, both
//     successors, MPS), so a state change is one table load;
//   * the candidate columns of a stripe are scanned as two 32-bit masks;
//   * all 32 lanes run the decoder in lock-step (replicated MQ state,
//     broadcast shared-memory accesses); at every stripe the lanes find the
//     candidate columns of the pass with __ballot_sync and the serial loop
//     visits only those; refinement contexts are precomputed by the lanes;
//   * the MQ byte stream is software-pipelined one byte ahead;
//   * the pass loop honours the coding-pass count (defect D3 fixed) and
//     updates the state it reads (defects D1/D2 fixed); every codeword byte is
//     consumed (defect D22 fixed) and one-column blocks stay in bounds (D23);
//   * the epilogue writes the block out coalesced with the inverse quantiser
//     fused in (ISO E.1, reconstruction point r);
//   * code-blocks with a coding style (bypass, context reset, termination on
//     every pass, vertically causal contexts, segmentation symbols; ISO
//     D.4-D.7) run in a launch of their own, an instantiation of the same
//     decoder that switches codeword segments at pass boundaries; the
//     reference decodes style 0 only.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <type_traits>

#include "t1_common.cuh"
#include "tc_internal.cuh"

namespace tc {
namespace {

#ifndef TC_T1_BLOCKS8
#define TC_T1_BLOCKS8 12
#endif
constexpr int kBlocks8 = TC_T1_BLOCKS8;  // code-blocks per CTA of the 8-bit class

// Blocks of more than 8 coded bit-planes keep their magnitude bits in their
// own output words instead of shared memory (OM, "output magnitudes"), so
// their state is smaller than an 8-bit block's and 24 warps of them reside
// per SM instead of 16 (with 4-block CTAs: lossless 12-bit 4096^2 Tier-1
// 48.7 -> 42.0 ms).  8-bit blocks keep them in shared memory, which is
// faster for them.  A launch too small to fill the GPU keeps them in shared
// memory too (OM false): each of its warps then runs nearly alone, and the
// output-word path's longer per-block latency would show (the 200,000-block
// workload decoded one launch per image: 1366 ms against 1049 ms).
template <typename MagT>
constexpr bool kOutMag = sizeof(MagT) > 1;

template <typename MagT, bool OM = kOutMag<MagT>>
struct WarpState {
    uint32_t F[kMaxStripes * 64];          // flag word per stripe column (with signs, bits 26-31)
    uint32_t ctx[20];                      // packed probability state per context
    uint8_t mrow[64];                      // refinement pass: rows of the stripe to refine
    uint8_t mctx[64];                      // refinement pass: 2-bit context code per row
    MagT mag[OM ? 4 : 64 * 64];            // magnitude bits decoded so far (unless OM)
};

// Signs in the decoder's flag word: bit 26 + j holds the sign of row j - 1 of
// the stripe column (j = 0..5, rows -1..4), set when that row becomes
// significant; rows -1 and 4 belong to the stripes above and below.
constexpr int kSignShift = 26;

// Sign-coding index (ISO Table D.3 neighbourhood) of row k of the column at
// F[i], whose flag word is f and 3x3 neighbourhood n9: the signs of the rows
// above and below come from f, those of the left and right neighbours from
// their own words.  Bits: up sign 0, up 1, left sign 2, left 3, right sign 4,
// right 5, down sign 6, down 7.
__device__ __forceinline__ uint32_t dec_sign_index(const uint32_t *F, uint32_t f, uint32_t n9, int i, int k, int c,
                                                   int w)
{
    const uint32_t lf = c > 0 ? F[i - 1] : 0u, rt = c + 1 < w ? F[i + 1] : 0u;
    const int own = kSignShift + 1 + k;  // this row's sign bit in a word of its stripe
    return (n9 & 0xAAu) | ((f >> (own - 1)) & 1u) | (((lf >> own) & 1u) << 2) | (((rt >> own) & 1u) << 4) |
           (((f >> (own + 1)) & 1u) << 6);
}

// Row k of stripe s in column c became significant with sign neg: the flag
// words of the neighbouring columns see its significance, and those of the
// stripes above and below also its sign.  The caller sets the column's own
// significance and sign bits.  With vertically causal contexts (vsc, ISO
// D.7) the stripe above does not see it: its last row's neighbourhood then
// leaves out the row below for every context.
__device__ __forceinline__ void dec_mark_significant(uint32_t *F, int s, int k, int c, int w, int nstripes,
                                                     uint32_t neg, bool vsc)
{
    const int i = s * 64 + c;
    if (c > 0) F[i - 1] |= 1u << (3 * k + 5);
    if (c + 1 < w) F[i + 1] |= 1u << (3 * k + 3);
    if (k == 0 && s > 0 && !vsc) {
        const int u = i - 64;
        F[u] |= (1u << 16) | (neg << (kSignShift + 5));
        if (c > 0) F[u - 1] |= 1u << 17;
        if (c + 1 < w) F[u + 1] |= 1u << 15;
    }
    if (k == 3 && s + 1 < nstripes) {
        const int d = i + 64;
        F[d] |= (1u << 1) | (neg << kSignShift);
        if (c > 0) F[d - 1] |= 1u << 2;
        if (c + 1 < w) F[d + 1] |= 1u << 0;
    }
}

// MQ decoder (ISO C.3; bytein/renormd/mqDecode, coefficient_coder.cl:121-252).
// The interval register A is kept scaled by 2^16 so that it lives in the same
// bit positions as C's upper half: the Qe comparison against C, the
// "A < 0x8000" test (sign bit of the scaled A) and the renormalisation shift
// (count of leading zeros) need no extra shifts.  Each context word is an
// entry of Tables::mqd: Qe << 16, the entries of its two successor states
// (after an MPS, after an LPS with the MPS switched where ISO Table C.2 says
// so) and the MPS in bit 0.  The byte after the current one is loaded ahead
// of use.
struct MQ {
    const uint8_t *p;
    int len, bp, ct;
    uint32_t a, c, cur, nxt;

    __device__ __forceinline__ uint32_t byte_at(int i) const { return i < len ? (uint32_t)__ldg(p + i) : 0xFFu; }
    __device__ __forceinline__ void bytein()
    {
        if (cur == 0xFF) {
            if (nxt > 0x8F) {
                c += 0xFF00;  // marker (or past the end): feed 1-bits, do not advance
                ct = 8;
                return;
            }
            c += nxt << 9;
            ct = 7;
        } else {
            c += nxt << 8;
            ct = 8;
        }
        bp++;
        cur = nxt;
        nxt = byte_at(bp + 1);   // used about nine decisions later: no prefetch needed
    }
    __device__ __forceinline__ void init(const uint8_t *d, int n)
    {
        p = d;
        len = n;
        bp = 0;
        cur = byte_at(0);
        nxt = byte_at(1);
        c = cur << 16;
        bytein();
        c <<= 7;
        ct -= 7;
        a = 0x80000000u;
    }
    __device__ __forceinline__ void renorm()
    {
        int sh = __clz(a);
        while (sh > ct) {
            a <<= ct;
            c <<= ct;
            sh -= ct;
            bytein();
        }
        a <<= sh;
        c <<= sh;
        ct -= sh;
    }
    // One decision.  The interval arithmetic of ISO C.3.2 (both the MPS and
    // the LPS sub-interval, with the conditional exchange) is done with
    // selects; the one branch left is the renormalisation, which is also
    // where the context's state moves on.
    __device__ __forceinline__ uint32_t decode(uint32_t *ctx, const uint32_t *tbl, int cx)
    {
        const uint32_t w = ctx[cx];
        const uint32_t qs = w & 0xFFFF0000u, mps = w & 1u;
        const uint32_t a1 = a - qs;
        const bool lower = c < qs;   // the code value lies in the Qe sub-interval
        const bool exch = a1 < qs;   // the conditional exchange swaps the symbols
        const uint32_t d = mps ^ (uint32_t)(lower != exch);
        c = lower ? c : c - qs;
        a = lower ? qs : a1;
        if (lower || (int)a1 >= 0) {
            ctx[cx] = tbl[d != mps ? (w >> 7) & 127u : w & 127u];
            renorm();
        }
        return d;
    }
};

// Raw (bypass) bits of ISO D.6: MSB first; a byte after 0xFF holds 7 bits
// (its MSB is a stuffed 0); after 0xFF a byte above 0x8F is a marker that is
// not consumed, and from there on (as past the end) 1-bits are read.
struct RawBits {
    const uint8_t *p;
    int len, bp, ct;
    uint32_t b;

    __device__ __forceinline__ void init(const uint8_t *d, int n)
    {
        p = d;
        len = n;
        bp = 0;
        ct = 0;
        b = 0;
    }
    __device__ __forceinline__ uint32_t bit()
    {
        if (ct == 0) {
            const uint32_t nb = bp < len ? (uint32_t)__ldg(p + bp) : 0xFFu;
            if (b == 0xFF && nb > 0x8F) {
                ct = 8;
            } else {
                ct = b == 0xFF ? 7 : 8;
                b = nb;
                bp++;
            }
        }
        --ct;
        return (b >> ct) & 1u;
    }
};

// Decode one code-block.  Every lane of the warp runs this function in
// lock-step; lanes split the per-stripe candidate searches between them
// (lane l owns columns l and l+32) and the serial loop visits only candidate
// columns, in scan order.  Returns the last pass type (0 cleanup,
// 1 significance propagation, 2 refinement) and its plane.
// Modes: the code-block style `style` applies; lens, when not null, holds
// the lengths of the codeword's terminated segments (BYPASS / TERMALL),
// which follow one another from seg.
// Raw: the block has raw (bypass) passes (BYPASS and more than 10 passes);
// without them the raw coder and its tests are compiled out.
template <typename MagT, int G, bool Modes = false, bool Raw = false, bool OM = kOutMag<MagT>>
__device__ int decode_block(WarpState<MagT, OM> &S, const Tables &T, const uint8_t *seg, int len, int w,
                            int h, int orient, int numbps, int passes, int *last_plane, int lane, unsigned gmask,
                            int gshift, uint32_t *ob, uint32_t pitch, int style = 0, const uint32_t *lens = nullptr)
{
    // magnitude bits: in shared memory, or (deep blocks) in the block's own
    // output words ob (row pitch `pitch`), where lane 0 of the group stores a
    // sample's first bit and ORs refinement bits in with fire-and-forget
    // atomics; the epilogue reads them back
    auto mag_set = [&](int y, int c, uint32_t v) {
        if constexpr (OM) {
            if (lane == 0) ob[(size_t)y * pitch + c] = v;
        } else {
            S.mag[y * 64 + c] = (MagT)v;
        }
    };
    auto mag_or = [&](int y, int c, uint32_t v) {
        if constexpr (OM) {
            if (lane == 0) atomicOr(ob + (size_t)y * pitch + c, v);
        } else {
            S.mag[y * 64 + c] |= (MagT)v;
        }
    };
    MQ mq;
    RawBits rw;
    bool raw = false;      // the current segment is raw-coded
    int segi = 0;          // current segment
    uint32_t segoff = 0;   // its first byte
    const bool vsc = Modes && (style & TC_CBLK_STYLE_VSC);
    if (!Modes || !lens) mq.init(seg, len);
    uint32_t *ctx = S.ctx;
    const uint32_t *tbl = T.mqd;
    const uint8_t *zc = T.zc[orient];
    uint32_t *F = S.F;
    const int nstripes = (h + 3) >> 2;
    constexpr int CPL = 64 / G;  // columns per lane
    int type = 0, pass = 0;
    *last_plane = numbps - 1;

    // before coding pass t: the next codeword segment starts where the
    // previous pass ended one
    auto begin_pass = [&](int t) {
        if constexpr (Modes) {
            if (!lens || (t > 0 && !style_pass_terminates(style, t - 1))) return;
            if (t > 0) segoff += lens[segi++];
            if constexpr (Raw) {
                raw = style_pass_raw(style, t);
                if (raw) {
                    rw.init(seg + segoff, (int)lens[segi]);
                    return;
                }
            }
            mq.init(seg + segoff, (int)lens[segi]);
        }
    };
    // after a pass: the contexts start over (RESET)
    auto end_pass = [&]() {
        if constexpr (Modes) {
            if (style & TC_CBLK_STYLE_RESET) {
                __syncwarp(gmask);
                for (int i = lane; i < 19; i += G)
                    ctx[i] = tbl[2 * (i == 0 ? 4 : (i == 17 ? 46 : (i == 18 ? 3 : 0)))];
                __syncwarp(gmask);
            }
        }
    };
    // one decision of a significance or refinement pass, and a sign
    auto decide = [&](int cx) -> uint32_t {
        if constexpr (Raw) {
            if (raw) return rw.bit();
        }
        return mq.decode(ctx, tbl, cx);
    };
    auto sign = [&](uint32_t si) -> uint32_t {
        if constexpr (Raw) {
            if (raw) return rw.bit();
        }
        return (uint32_t)mq.decode(ctx, tbl, si & 15) ^ (si >> 4);
    };

    for (int p = numbps - 1; p >= 0; --p) {
        const uint32_t pbit = 1u << p;
        if (p != numbps - 1) {
            // ---- significance propagation pass (ISO D.3.1; SigPropPassFunctor) ----
            begin_pass(pass);
            for (int s = 0; s < nstripes; s++) {
                const int rows = min(4, h - 4 * s);
                __syncwarp(gmask);
                bool any[CPL];
#pragma unroll
                for (int j = 0; j < CPL; j++) {
                    const int c = lane + G * j;
                    bool a = false;
                    if (c < w) {
                        // bit 3j of g: a significant sample in row j - 1 of
                        // the three columns; bit 3k of the test: row k is not
                        // significant and has a significant neighbour
                        const uint32_t f = F[s * 64 + c];
                        const uint32_t g = (f | (f >> 1) | (f >> 2)) & 0x9249u;
                        a = ((g | (g >> 3) | (g >> 6)) & ~(f >> 4) & (0x249u >> (3 * (4 - rows)))) != 0u;
                    }
                    any[j] = a;
                }
                const unsigned long long cand64 = group_ballot<G>(any, gmask, gshift);
                uint32_t chi = (uint32_t)(cand64 >> 32);  // columns 32-63
#pragma unroll 1
                for (int half = 0; half < 2; half++) {
                    uint32_t cand = half ? chi : (uint32_t)cand64;
                    while (cand) {
                        const int c = 32 * half + __ffs(cand) - 1;
                        cand &= cand - 1;
                        uint32_t f = F[s * 64 + c];
                        for (int k = 0; k < rows; k++) {
                            const uint32_t fk = f >> (3 * k);   // row k's window at bit 0, self at bit 4
                            if (fk & 0x10u) continue;
                            const uint32_t n9 = fk & 0x1FFu;
                            if (!(n9 & 0x1EFu)) continue;
                            f |= pi_bit(k);
                            if (decide(zc[n9])) {
                                const uint32_t si = T.sc[dec_sign_index(F, f, n9, s * 64 + c, k, c, w)];
                                const uint32_t neg = sign(si);
                                f |= self_bit(k) | (neg << (kSignShift + 1 + k));
                                dec_mark_significant(F, s, k, c, w, nstripes, neg, vsc);
                                mag_set(4 * s + k, c, pbit);
                                if (c + 1 < w) {  // the next column gained a neighbour
                                    cand |= 2u << (c & 31);
                                    chi |= (uint32_t)(c == 31);
                                }
                            }
                        }
                        // stored unconditionally: a visited column nearly
                        // always had a row coded (its pi bit set)
                        F[s * 64 + c] = f;
                    }
                }
            }
            end_pass();
            type = 1;
            *last_plane = p;
            if (++pass >= passes) break;

            // ---- magnitude refinement pass (ISO D.3.3; MagRefPassFunctor) ----
            // Rows to refine and their contexts do not change during the pass:
            // the lanes precompute them for their columns.
            begin_pass(pass);
            for (int s = 0; s < nstripes; s++) {
                const int rows = min(4, h - 4 * s);
                __syncwarp(gmask);
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
                const unsigned long long cand64 = group_ballot<G>(any, gmask, gshift);
                __syncwarp(gmask);
#pragma unroll 1
                for (int half = 0; half < 2; half++) {
                    uint32_t cand = half ? (uint32_t)(cand64 >> 32) : (uint32_t)cand64;
                    while (cand) {
                        const int c = 32 * half + __ffs(cand) - 1;
                        cand &= cand - 1;
                        uint32_t rr = S.mrow[c];
                        const uint32_t codes = S.mctx[c];
                        while (rr) {
                            const int k = __ffs(rr) - 1;
                            rr &= rr - 1;
                            if (decide(14 + ((codes >> (2 * k)) & 3u))) mag_or(4 * s + k, c, pbit);
                        }
                    }
                }
            }
            end_pass();
            type = 2;
            if (++pass >= passes) break;
        }

        // ---- cleanup pass (ISO D.3.4; CleanUpPassFunctor) ----
        begin_pass(pass);
        for (int s = 0; s < nstripes; s++) {
            const int rows = min(4, h - 4 * s);
            const uint32_t rmask = (1u << rows) - 1u;
            __syncwarp(gmask);
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
            const unsigned long long cand64 = group_ballot<G>(any, gmask, gshift);
#pragma unroll 1
            for (int half = 0; half < 2; half++) {
                uint32_t cand = half ? (uint32_t)(cand64 >> 32) : (uint32_t)cand64;
                while (cand) {
                    const int c = 32 * half + __ffs(cand) - 1;
                    cand &= cand - 1;
                    uint32_t f = F[s * 64 + c];
                    const uint32_t f0 = f;
                    int k = 0;
                    if (rows == 4 && (f & kSigMask) == 0u) {
                        // run-length mode: four rows with an all-zero neighbourhood
                        if (!mq.decode(ctx, tbl, 18)) continue;
                        int r = mq.decode(ctx, tbl, 17) << 1;
                        r |= mq.decode(ctx, tbl, 17);
                        const uint32_t si = T.sc[dec_sign_index(F, f, (f >> (3 * r)) & 0x1FFu, s * 64 + c, r, c, w)];
                        const uint32_t neg = (uint32_t)mq.decode(ctx, tbl, si & 15) ^ (si >> 4);
                        f |= self_bit(r) | (neg << (kSignShift + 1 + r));
                        dec_mark_significant(F, s, r, c, w, nstripes, neg, vsc);
                        mag_set(4 * s + r, c, pbit);
                        k = r + 1;
                    }
                    for (; k < rows; k++) {
                        if (f & (self_bit(k) | pi_bit(k))) continue;
                        const uint32_t n9 = (f >> (3 * k)) & 0x1FFu;
                        if (mq.decode(ctx, tbl, zc[n9])) {
                            const uint32_t si = T.sc[dec_sign_index(F, f, n9, s * 64 + c, k, c, w)];
                            const uint32_t neg = (uint32_t)mq.decode(ctx, tbl, si & 15) ^ (si >> 4);
                            f |= self_bit(k) | (neg << (kSignShift + 1 + k));
                            dec_mark_significant(F, s, k, c, w, nstripes, neg, vsc);
                            mag_set(4 * s + k, c, pbit);
                        }
                    }
                    if (f != f0) F[s * 64 + c] = f;
                }
            }
        }
        if constexpr (Modes) {
            if (style & TC_CBLK_STYLE_SEGSYM)  // segmentation symbol 1010 (ISO D.5)
                for (int i = 0; i < 4; i++) mq.decode(ctx, tbl, 17);
        }
        end_pass();
        type = 0;
        *last_plane = p;
        if (++pass >= passes) break;
        __syncwarp(gmask);
        for (int i = lane; i < nstripes * 64; i += G) F[i] &= ~0x3C0000u;  // clear pi
        __syncwarp(gmask);
    }
    return type;
}

// Lanes per code-block G (32, 16 or 8): a warp splits into 32 / G groups that
// decode different code-blocks in lock-step (each group runs the serial
// decoder redundantly across its lanes and splits the candidate searches
// between them), so one warp instruction can advance several code-blocks.
// Code-blocks per CTA: the per-CTA label tables are shared by more blocks
// when the block state is small, which lets more warps reside per SM (8-bit
// state: 2 CTAs of 12 blocks = 24 per SM within 228 KB, against 5 CTAs of 4).
// Register budget (min_ctas, the launch bound's minimum CTAs per SM): the
// plain instantiations leave the count to the compiler (1), which gives the
// 8-bit kernel 76 registers, still two 384-thread CTAs per SM; against the
// 64 it picks when told to expect more CTAs, that is 7.5% faster on the
// 4096^2 workload (and 12 blocks per CTA beat 8 at the same count by 5%).
// The styled instantiations use more registers, so they are told how many
// CTAs their shared memory lets reside, which keeps that occupancy.
template <typename MagT, int G, bool OM = kOutMag<MagT>>
struct GroupCfg {
    static constexpr int blocks = sizeof(MagT) == 1 ? kBlocks8 : 4;
    static constexpr int warps = blocks * G / 32 > 0 ? blocks * G / 32 : 1;
    static constexpr size_t smem =
        ((sizeof(Tables) + 15) & ~size_t(15)) + (size_t)blocks * sizeof(WarpState<MagT, OM>);
    static constexpr int by_smem = (int)((228u * 1024u) / (smem + 1024u));
    static constexpr int by_warps = 24 / warps < 1 ? 1 : 24 / warps;   // 24 warps per SM
    template <bool Modes>
    static constexpr int min_ctas() { return Modes ? (by_smem < 1 ? 1 : (by_smem > by_warps ? by_warps : by_smem)) : 1; }
};

// Decode code-block `bi` with the state S and write it out (the group's
// lanes, in lock-step).  MagT bounds the coded bit-planes it accepts.
template <typename MagT, int G, bool Modes = false, bool OM = kOutMag<MagT>>
__device__ __forceinline__ void process_block(WarpState<MagT, OM> &S, const Tables &T, const tc_cblk_desc *__restrict__ desc,
                                              uint32_t bi, int ndesc, const uint8_t *__restrict__ pool,
                                              uint64_t pool_len, char *__restrict__ out, uint64_t out_elems, int out_mode,
                                              float recon_r, uint32_t *__restrict__ err, int gl, unsigned gmask,
                                              int gshift)
{
    if (bi >= (uint32_t)ndesc) {
        if (gl == 0) atomicOr(err, TC_DERR_DESC);
        return;
    }
    const tc_cblk_desc d = desc[bi];
    const int w = d.w, h = d.h;
    const bool geom_ok = w >= 1 && w <= 64 && h >= 1 && h <= 64;
    const int numbps = (int)d.mb - (int)d.zero_bitplanes;
    bool ok = geom_ok && d.mb >= 1 && d.mb <= 31 && d.orient <= 3 && numbps >= 0 &&
              (numbps == 0 || d.passes <= 3 * numbps - 2) && numbps <= (int)(8 * sizeof(MagT));
    const bool pool_ok = d.seg_off <= pool_len && (uint64_t)d.seg_len <= pool_len - d.seg_off;
    if (!geom_ok) {
        if (gl == 0) atomicOr(err, TC_DERR_DESC);
        return;
    }
    // the block's last sample, out_off + (h-1) * out_pitch + w - 1, must lie
    // inside the output; a block that does not is skipped before any write
    if (d.out_off > out_elems || (uint64_t)(h - 1) * d.out_pitch + (uint64_t)w > out_elems - d.out_off) {
        if (gl == 0) atomicOr(err, TC_DERR_OUT);
        return;
    }
    if (!ok || !pool_ok) {
        if (gl == 0) atomicOr(err, ok ? TC_DERR_POOL : TC_DERR_DESC);
        ok = false;
    }
    // Styled blocks: only the Modes launch decodes them.  A segment table
    // (BYPASS / TERMALL) sits 4-byte aligned at seg_off, the codeword after
    // it, and its lengths add up to seg_len.
    const int style = d.style & kStyleDecodeBits;
    const uint32_t *lens = nullptr;
    uint64_t cw_off = d.seg_off;
    if (!Modes && style) {
        if (gl == 0) atomicOr(err, TC_DERR_STYLE);
        ok = false;
    }
    if (Modes && ok && (style & (TC_CBLK_STYLE_BYPASS | TC_CBLK_STYLE_TERMALL)) && numbps > 0 && d.passes > 0) {
        const int nseg = style_segments(style, d.passes);
        const uint64_t tab = 4ull * (uint64_t)nseg;
        bool tab_ok = (d.seg_off & 3u) == 0 && d.seg_off + tab <= pool_len &&
                      (uint64_t)d.seg_len <= pool_len - d.seg_off - tab;
        if (tab_ok) {
            lens = reinterpret_cast<const uint32_t *>(pool + d.seg_off);
            uint64_t sum = 0;
            for (int i = 0; i < nseg; i++) sum += __ldg(lens + i);
            tab_ok = sum == d.seg_len;
            cw_off += tab;
        }
        if (!tab_ok) {
            if (gl == 0) atomicOr(err, TC_DERR_STYLE);
            ok = false;
        }
    }
    const bool coded = ok && numbps > 0 && d.passes > 0;
    const int nstripes = (h + 3) >> 2;

    // clear the state (the group's lanes)
    for (int i = gl; i < nstripes * 64; i += G) S.F[i] = 0u;
    for (int i = gl; i < 19; i += G) {
        const int st = i == 0 ? 4 : (i == 17 ? 46 : (i == 18 ? 3 : 0));
        S.ctx[i] = T.mqd[2 * st];   // MPS 0
    }
    __syncwarp(gmask);

    int type = 0, last_plane = 0;
    uint32_t *ob = reinterpret_cast<uint32_t *>(out) + d.out_off;   // the block's output words
    if (coded) {
        if (Modes && (style & TC_CBLK_STYLE_BYPASS) && d.passes > 10)
            type = decode_block<MagT, G, Modes, Modes, OM>(S, T, pool + cw_off, (int)d.seg_len, w, h, d.orient, numbps,
                                                       d.passes, &last_plane, gl, gmask, gshift, ob, d.out_pitch, style,
                                                       lens);
        else
            type = decode_block<MagT, G, Modes, false, OM>(S, T, pool + cw_off, (int)d.seg_len, w, h, d.orient, numbps,
                                                       d.passes, &last_plane, gl, gmask, gshift, ob, d.out_pitch, style,
                                                       lens);
    }
    if constexpr (OM) __threadfence();   // lane 0's magnitude writes, before the group reads them
    __syncwarp(gmask);

    // epilogue: reconstruction + inverse quantisation, coalesced rows; an
    // ROI magnitude (>= 2^roi) is shifted down by roi (ISO H.1), and so is
    // its count of undecoded planes
    const bool irrev = (d.flags & TC_CBLK_IRREVERSIBLE) != 0;
    const int roi = d.roi_shift < d.mb ? d.roi_shift : 0;
    const int mb_out = d.mb - roi;  // magnitude bits after the ROI shift
    for (int y = 0; y < h; y++) {
        char *row = out + 4 * (d.out_off + (uint64_t)y * d.out_pitch);
        const int s = y >> 2, k = y & 3;
        for (int x = gl; x < w; x += G) {
            const uint32_t f = coded ? S.F[s * 64 + x] : 0u;
            const bool sg = (f & self_bit(k)) != 0u;
            uint32_t mg = 0, neg = 0, u = 0;
            if (sg) {
                if constexpr (OM)
                    mg = __ldcg(reinterpret_cast<const uint32_t *>(row) + x);
                else
                    mg = (uint32_t)S.mag[y * 64 + x];
                neg = (f >> (kSignShift + 1 + k)) & 1u;
                u = (uint32_t)last_plane;
                if (type == 1 && !(f & pi_bit(k))) u++;
                if (roi && (mg >> roi)) {
                    mg >>= roi;
                    u = u > (uint32_t)roi ? u - roi : 0u;
                }
            }
            if (out_mode == TC_T1_OUT_RAW) {
                reinterpret_cast<uint32_t *>(row)[x] = sg ? ((mg << (31 - mb_out)) | (neg << 31)) : 0u;
            } else if (irrev) {
                float v = 0.0f;
                if (sg) v = ((float)mg + recon_r * (float)(1u << u)) * d.step;
                reinterpret_cast<float *>(row)[x] = neg ? -v : v;
            } else {
                int32_t v = 0;
                if (sg) v = (int32_t)mg + (u ? (int32_t)floorf(recon_r * (float)(1u << u)) : 0);
                reinterpret_cast<int32_t *>(row)[x] = neg ? -v : v;
            }
        }
    }
    __syncwarp(gmask);
}

// Persistent Tier-1 launch over one magnitude class.  The 8-bit class with
// 32-lane groups can also take a short queue of 16-bit blocks (`heavy`): in
// each of the first `heavy_ctas` CTAs warp 0 becomes a 16-bit decoder in
// its own state slot (a deep block's magnitudes live in its output words),
// drains the heavy queue first and then joins the 8-bit queue.  A few blocks with many
// bit-planes thus start at once, one per CTA, in the same longest-first
// launch as the bulk, instead of running as a separate class whose warps
// share SMs with the bulk and become the launch's longest chain.
struct HeavyQueue {
    const uint32_t *order = nullptr;
    int n = 0;
    int ctas = 0;
    uint32_t *counter = nullptr;
};

template <typename MagT, int G, bool Modes = false, bool OM = kOutMag<MagT>>
__global__ void __launch_bounds__(32 * GroupCfg<MagT, G, OM>::warps, GroupCfg<MagT, G, OM>::template min_ctas<Modes>())
t1_decode_kernel(const tc_cblk_desc *__restrict__ desc, const uint32_t *__restrict__ order, int n, int ndesc,
                 const uint8_t *__restrict__ pool, uint64_t pool_len, char *__restrict__ out, uint64_t out_elems,
                 int out_mode, float recon_r, uint32_t *__restrict__ counter, uint32_t *__restrict__ err, HeavyQueue heavy)
{
    extern __shared__ __align__(16) unsigned char smem[];
    Tables &T = *reinterpret_cast<Tables *>(smem);
    WarpState<MagT, OM> *states =
        reinterpret_cast<WarpState<MagT, OM> *>(smem + ((sizeof(Tables) + 15) & ~size_t(15)));
    build_tables(T);
    __syncthreads();

    const int wl = threadIdx.x & 31;             // lane in the warp
    const int gidx = wl / G, gl = wl % G;         // group in the warp, lane in the group
    const int gshift = gidx * G;
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << gshift);
    const int slot = (threadIdx.x >> 5) * (32 / G) + gidx;
    WarpState<MagT, OM> &S = states[slot];

    if constexpr (std::is_same<MagT, uint8_t>::value && G == 32) {
        static_assert(sizeof(WarpState<uint16_t>) <= sizeof(WarpState<uint8_t>), "heavy state fits a slot");
        if ((int)blockIdx.x < heavy.ctas && slot == 0) {
            WarpState<uint16_t> &HS = *reinterpret_cast<WarpState<uint16_t> *>(&states[0]);
            for (;;) {
                int idx = 0;
                if (wl == 0) idx = (int)atomicAdd(heavy.counter, 1u);
                idx = __shfl_sync(0xffffffffu, idx, 0);
                if (idx >= heavy.n) break;
                process_block<uint16_t, 32, Modes>(HS, T, desc, heavy.order[idx], ndesc, pool, pool_len, out,
                                                   out_elems, out_mode, recon_r, err, gl, gmask, gshift);
            }
        }
    }

    for (;;) {
        int idx = 0;
        if (gl == 0) idx = (int)atomicAdd(counter, 1u);
        idx = __shfl_sync(gmask, idx, gshift);
        if (idx >= n) break;
        const uint32_t bi = order ? order[idx] : (uint32_t)idx;
        process_block<MagT, G, Modes, OM>(S, T, desc, bi, ndesc, pool, pool_len, out, out_elems, out_mode, recon_r, err, gl,
                                      gmask, gshift);
    }
}

// Standalone inverse quantiser over raw sign-magnitude words.
__global__ void dequant_raw_kernel(const tc_cblk_desc *__restrict__ desc, int n,
                                   const uint32_t *__restrict__ raw, char *__restrict__ out, uint64_t elems,
                                   float recon_r, uint32_t *words, bool base16)
{
    const int b = blockIdx.x;
    if (b >= n) return;
    const tc_cblk_desc d = desc[b];
    if (d.w < 1 || d.w > 64 || d.h < 1 || d.h > 64 || d.mb < 1 || d.mb > 31) {
        if (threadIdx.x == 0) atomicOr(&words[0], TC_DERR_DESC);
        return;
    }
    // raw words and output share the block's place: both hold `elems`
    if (d.out_off > elems || (uint64_t)(d.h - 1) * d.out_pitch + (uint64_t)d.w > elems - d.out_off) {
        if (threadIdx.x == 0) atomicOr(&words[0], TC_DERR_OUT);
        return;
    }
    const int numbps = (int)d.mb - (int)d.zero_bitplanes;
    const int roi = d.roi_shift < d.mb ? d.roi_shift : 0;
    const int mb = d.mb - roi;  // magnitude bits of the raw words
    // Decoded planes from the pass count: the last pass ran on plane p_last
    // (counted in the ROI-shifted domain for an ROI block).
    int u = 0;
    if (numbps > 0 && d.passes > 0) {
        const int p_last = numbps - 1 - (d.passes + 1) / 3 - roi;
        u = p_last < 0 ? 0 : p_last;
    }
    const bool irrev = (d.flags & TC_CBLK_IRREVERSIBLE) != 0;
    const float fr = recon_r * (float)(1u << u);
    const int32_t ir = u ? (int32_t)floorf(fr) : 0;
    // 16 threads per row, four consecutive coefficients each (one 16-byte
    // load and store when the block's rows are aligned): whole rows, no
    // index division
    auto one = [&](uint32_t r) -> uint32_t {
        const uint32_t mg = (r & 0x7FFFFFFFu) >> (31 - mb);
        const bool neg = (r >> 31) != 0;
        if (irrev) {
            const float v = mg ? ((float)mg + fr) * d.step : 0.0f;
            return __float_as_uint(neg ? -v : v);
        }
        const int32_t v = mg ? (int32_t)mg + ir : 0;
        return (uint32_t)(neg ? -v : v);
    };
    const int x = 4 * (threadIdx.x & 15);
    if (x >= d.w) return;
    const bool vec = base16 && ((d.out_off | (uint64_t)d.out_pitch) & 3u) == 0 && x + 4 <= d.w;
    uint32_t *dst = reinterpret_cast<uint32_t *>(out);
    for (int y = threadIdx.x >> 4; y < d.h; y += blockDim.x >> 4) {
        const uint64_t o = d.out_off + (uint64_t)y * d.out_pitch + x;
        if (vec) {
            const uint4 r = *reinterpret_cast<const uint4 *>(raw + o);
            *reinterpret_cast<uint4 *>(dst + o) = make_uint4(one(r.x), one(r.y), one(r.z), one(r.w));
        } else {
            for (int j = 0; j < 4 && x + j < d.w; j++) dst[o + j] = one(raw[o + j]);
        }
    }
}

struct LaunchCfg {
    int per_sm = 1;    // resident CTAs per SM
    int per_cta = 4;   // code-blocks in flight per CTA
    size_t smem = 0;   // dynamic shared memory per CTA
};

// Kernel attributes and occupancy of one class variant, set up once per device.
template <typename MagT, int G, bool Modes = false, bool OM = kOutMag<MagT>>
cudaError_t class_cfg(tc_ctx *ctx, LaunchCfg **out)
{
    constexpr int kWarps = GroupCfg<MagT, G, OM>::warps;
    static LaunchCfg cfg[64];
    static DeviceFlags ready;
    LaunchCfg &C = cfg[ctx->device & 63];
    const cudaError_t e = once_per_device(ready, ctx->device, [&] {
        C.smem = ((sizeof(Tables) + 15) & ~size_t(15)) + kWarps * (32 / G) * sizeof(WarpState<MagT, OM>);
        C.per_cta = kWarps * (32 / G);
        cudaError_t r = cudaFuncSetAttribute(t1_decode_kernel<MagT, G, Modes, OM>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C.smem);
        if (r == cudaSuccess)
            r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&C.per_sm, t1_decode_kernel<MagT, G, Modes, OM>,
                                                              32 * kWarps, C.smem);
        if (C.per_sm < 1) C.per_sm = 1;
        return r;
    });
    *out = &C;
    return e;
}

// One class launch: a persistent grid pulling the class's blocks from its
// work counter d_words[slot] (zeroed beforehand).
template <typename MagT, int G, bool Modes = false, bool OM = kOutMag<MagT>>
cudaError_t launch_class_om(tc_ctx *ctx, cudaStream_t stream, const tc_cblk_desc *d_desc, const uint32_t *d_order,
                            int n, int ndesc, const uint8_t *d_pool, uint64_t pool_len, void *d_out, uint64_t out_elems,
                            int out_mode, float recon_r, int slot, const HeavyQueue &heavy = HeavyQueue())
{
    LaunchCfg *C = nullptr;
    cudaError_t e = class_cfg<MagT, G, Modes, OM>(ctx, &C);
    if (e != cudaSuccess) return e;
    const int want = std::max((n + C->per_cta - 1) / C->per_cta, heavy.ctas);
    const int grid = std::max(1, std::min(want, C->per_sm * num_sms(ctx->device)));
    t1_decode_kernel<MagT, G, Modes, OM><<<grid, 32 * GroupCfg<MagT, G, OM>::warps, C->smem, stream>>>(
        d_desc, d_order, n, ndesc, d_pool, pool_len, static_cast<char *>(d_out), out_elems, out_mode, recon_r,
        ctx->d_words + slot, ctx->d_words, heavy);
    ctx->launches++;
    return cudaGetLastError();
}

// A 32-lane launch of a deep class keeps its magnitudes in the output words
// only when its blocks fill the GPU (one block for each of 24 warps on every
// SM); a smaller one keeps them in shared memory.
template <typename MagT, int G, bool Modes = false>
cudaError_t launch_class(tc_ctx *ctx, cudaStream_t stream, const tc_cblk_desc *d_desc, const uint32_t *d_order,
                         int n, int ndesc, const uint8_t *d_pool, uint64_t pool_len, void *d_out, uint64_t out_elems,
                         int out_mode, float recon_r, int slot, const HeavyQueue &heavy = HeavyQueue())
{
    if constexpr (kOutMag<MagT> && G == 32) {
        if (n < 24 * num_sms(ctx->device))
            return launch_class_om<MagT, G, Modes, false>(ctx, stream, d_desc, d_order, n, ndesc, d_pool, pool_len, d_out,
                                                          out_elems, out_mode, recon_r, slot, heavy);
    }
    return launch_class_om<MagT, G, Modes>(ctx, stream, d_desc, d_order, n, ndesc, d_pool, pool_len, d_out, out_elems,
                                           out_mode, recon_r, slot, heavy);
}

template <typename MagT>
cudaError_t launch_class_g(tc_ctx *ctx, cudaStream_t stream, const tc_cblk_desc *d_desc, const uint32_t *d_order,
                           int n, int ndesc, const uint8_t *d_pool, uint64_t pool_len, void *d_out, uint64_t out_elems, int out_mode,
                           float recon_r, int slot)
{
    switch (ctx->t1_group) {
    case 8:
        return launch_class<MagT, 8>(ctx, stream, d_desc, d_order, n, ndesc, d_pool, pool_len, d_out, out_elems, out_mode,
                                     recon_r, slot);
    case 16:
        return launch_class<MagT, 16>(ctx, stream, d_desc, d_order, n, ndesc, d_pool, pool_len, d_out, out_elems, out_mode,
                                      recon_r, slot);
    default:
        return launch_class<MagT, 32>(ctx, stream, d_desc, d_order, n, ndesc, d_pool, pool_len, d_out, out_elems, out_mode,
                                      recon_r, slot);
    }
}

// Largest 16-bit class that rides along in the 8-bit launch: one heavy
// decoder per CTA, so at most one CTA per SM gives up one warp, and only next
// to a bulk at least eight times larger.
constexpr int kMaxHeavy = 148;

}  // namespace

cudaError_t launch_t1_decode(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order, int n,
                             const uint8_t *d_pool, uint64_t pool_len, void *d_out, uint64_t out_elems, int out_mode, float recon_r,
                             int max_bitplanes)
{
    if (out_mode & TC_T1_STYLED) {
        const int s[3] = {max_bitplanes <= 8 ? n : 0, max_bitplanes > 8 && max_bitplanes <= 16 ? n : 0,
                          max_bitplanes > 16 ? n : 0};
        return launch_t1_classes(ctx, d_desc, d_order, n, 0, 0, 0, d_pool, pool_len, d_out, out_elems, out_mode & ~TC_T1_STYLED,
                                 recon_r, s);
    }
    return launch_t1_classes(ctx, d_desc, d_order, n, max_bitplanes <= 8 ? n : 0,
                             max_bitplanes > 8 && max_bitplanes <= 16 ? n : 0, max_bitplanes > 16 ? n : 0, d_pool,
                             pool_len, d_out, out_elems, out_mode, recon_r);
}

// Classes: blocks of <= 8, <= 16 and <= 31 coded bit-planes, in that order in
// d_order (each slice longest first).  A wider state decodes any narrower
// block, so a minority class joins its neighbour's launch: a short 16-bit
// class rides in the 8-bit launch (see HeavyQueue), and an 8-bit class at
// most half the size of the 16-bit class is decoded by the 16-bit launch.
// Otherwise the classes run as concurrent launches, the 32- and 16-bit ones
// on side streams.  Styled blocks (after the three classes, in the same
// three widths: nstyled[0..2]) run in Modes launches on the context's stream.
cudaError_t launch_t1_classes(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order, int ndesc,
                              int n8, int n16, int n32, const uint8_t *d_pool, uint64_t pool_len, void *d_out,
                              uint64_t out_elems, int out_mode, float recon_r, const int *nstyled)
{
    int ns8 = nstyled ? nstyled[0] : 0, ns16 = nstyled ? nstyled[1] : 0, ns32 = nstyled ? nstyled[2] : 0;
    if (n8 + n16 + n32 + ns8 + ns16 + ns32 == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(ctx->d_words + 1, 0, 6 * sizeof(uint32_t), ctx->stream);
    if (e != cudaSuccess) return e;
    if (ns8 + ns16 + ns32 > 0) {
        // the widths run concurrently (the wider ones on side streams), so
        // a few deep blocks start with the bulk instead of after it
        const uint32_t *os = d_order ? d_order + n8 + n16 + n32 : nullptr;
        // a short 16-bit class rides in the 8-bit launch, as for unstyled blocks
        HeavyQueue sheavy;
        if (ns8 > 0 && ns16 > 0 && ns16 <= kMaxHeavy && 8 * ns16 <= ns8 && os) {
            sheavy.order = os + ns8;
            sheavy.n = ns16;
            sheavy.ctas = ns16;
            sheavy.counter = ctx->d_words + 5;
            ns16 = 0;
        }
        const int nl = (ns8 > 0) + (ns16 > 0) + (ns32 > 0);
        cudaStream_t w8 = ctx->stream, w16 = ctx->stream, w32 = ctx->stream;
        if (nl > 1) {
            if ((e = ensure_side_streams(ctx)) != cudaSuccess) return e;
            if ((e = cudaEventRecord(ctx->ev_fork, ctx->stream)) != cudaSuccess) return e;
            for (int i = 0; i < 2; i++)
                if ((e = cudaStreamWaitEvent(ctx->side[i], ctx->ev_fork, 0)) != cudaSuccess) return e;
            w32 = ctx->side[0];
            w16 = ctx->side[1];
        }
        if (ns32 > 0)
            e = launch_class<uint32_t, 32, true>(ctx, w32, d_desc, os ? os + ns8 + ns16 : nullptr, ns32, ndesc, d_pool,
                                                 pool_len, d_out, out_elems, out_mode, recon_r, 6);
        if (e == cudaSuccess && ns16 > 0)
            e = launch_class<uint16_t, 32, true>(ctx, w16, d_desc, os ? os + ns8 : nullptr, ns16, ndesc, d_pool,
                                                 pool_len, d_out, out_elems, out_mode, recon_r, 5);
        if (e == cudaSuccess && ns8 > 0)
            e = launch_class<uint8_t, 32, true>(ctx, w8, d_desc, os, ns8, ndesc, d_pool, pool_len, d_out, out_elems, out_mode,
                                                recon_r, 4, sheavy);
        if (nl > 1) {
            for (int i = 0; i < 2; i++) {
                cudaError_t e2 = cudaEventRecord(ctx->ev_join[i], ctx->side[i]);
                if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(ctx->stream, ctx->ev_join[i], 0);
                if (e == cudaSuccess) e = e2;
            }
        }
        if (e != cudaSuccess || n8 + n16 + n32 == 0) return e;
    }
    const uint32_t *o16 = d_order ? d_order + n8 : nullptr;
    const uint32_t *o32 = d_order ? d_order + n8 + n16 : nullptr;
    HeavyQueue heavy;
    if (n8 > 0 && n16 > 0 && n16 <= kMaxHeavy && 8 * n16 <= n8 && d_order && ctx->t1_group == 32) {
        heavy.order = o16;
        heavy.n = n16;
        heavy.ctas = n16;
        heavy.counter = ctx->d_words + 2;
        n16 = 0;
    } else if (n8 > 0 && n16 > 0 && 2 * n8 <= n16 && d_order) {
        o16 = d_order;  // the 8-bit slice directly precedes the 16-bit one
        n16 += n8;
        n8 = 0;
    }
    const int nlaunch = (n8 > 0) + (n16 > 0) + (n32 > 0);
    cudaStream_t s8 = ctx->stream, s16 = ctx->stream, s32 = ctx->stream;
    if (nlaunch > 1) {
        // Fork: the heavier classes run on side streams, concurrently with
        // the 8-bit class on the context's stream, and are joined after it.
        if ((e = ensure_side_streams(ctx)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(ctx->ev_fork, ctx->stream)) != cudaSuccess) return e;
        for (int i = 0; i < 2; i++)
            if ((e = cudaStreamWaitEvent(ctx->side[i], ctx->ev_fork, 0)) != cudaSuccess) return e;
        s32 = ctx->side[0];
        s16 = ctx->side[1];
    }
    if (n32 > 0)
        e = launch_class_g<uint32_t>(ctx, s32, d_desc, o32, n32, ndesc, d_pool, pool_len, d_out, out_elems, out_mode,
                                     recon_r, 3);
    if (e == cudaSuccess && n16 > 0)
        e = launch_class_g<uint16_t>(ctx, s16, d_desc, o16, n16, ndesc, d_pool, pool_len, d_out, out_elems, out_mode,
                                     recon_r, 2);
    if (e == cudaSuccess && n8 > 0) {
        if (heavy.n > 0)
            e = launch_class<uint8_t, 32>(ctx, s8, d_desc, d_order, n8, ndesc, d_pool, pool_len, d_out, out_elems, out_mode,
                                          recon_r, 1, heavy);
        else
            e = launch_class_g<uint8_t>(ctx, s8, d_desc, d_order, n8, ndesc, d_pool, pool_len, d_out, out_elems, out_mode,
                                        recon_r, 1);
    }
    if (nlaunch > 1) {
        for (int i = 0; i < 2; i++) {
            cudaError_t e2 = cudaEventRecord(ctx->ev_join[i], ctx->side[i]);
            if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(ctx->stream, ctx->ev_join[i], 0);
            if (e == cudaSuccess) e = e2;
        }
    }
    return e;
}

cudaError_t launch_dequant_raw(tc_ctx *ctx, const tc_cblk_desc *d_desc, int n, const uint32_t *d_raw,
                               void *d_out, uint64_t elems, float recon_r)
{
    if (n <= 0) return cudaSuccess;
    const bool base16 = ((reinterpret_cast<uintptr_t>(d_raw) | reinterpret_cast<uintptr_t>(d_out)) & 15) == 0;
    dequant_raw_kernel<<<n, 256, 0, ctx->stream>>>(d_desc, n, d_raw, static_cast<char *>(d_out), elems, recon_r,
                                                   ctx->d_words, base16);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace tc
