// t1_common.cuh -- pieces shared by the Tier-1 decoder (t1_decode.cu) and
// encoder (t1_encode.cu): the flag-word layout of a code-block's state, the
// MQ probability-state table and the context-label tables (ISO Annex C.2,
// D.3).  Included inside namespace tc's anonymous namespace of each file.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tc_j2k.h"

namespace tc {
namespace {

constexpr int kMaxStripes = 16;    // 64 rows
constexpr int kSgnCols = 66;       // 64 columns + a zero column on each side

// Flag word layout (one per stripe column):
//   bits 0-17  significance, bit 3*j + col for row j-1 of the stripe
//              (j = 0..5, rows -1..4) and col 0 = left, 1 = this, 2 = right
//   bits 18-21 pi: coded in this plane's significance propagation pass
//   bits 22-25 sigma': refined at least once
//   bits 26-31 (decoder only) sign of row j-1 at bit 26 + j, j = 0..5
constexpr uint32_t kSigMask = 0x3FFFFu;
__device__ __forceinline__ uint32_t self_bit(int k) { return 1u << (3 * k + 4); }
__device__ __forceinline__ uint32_t pi_bit(int k) { return 1u << (18 + k); }
__device__ __forceinline__ uint32_t ref_bit(int k) { return 1u << (22 + k); }

// ISO Table C.2 (coefficient_coder.cl:36-60).
__constant__ uint16_t c_qe[47] = {
    0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801,
    0x3001, 0x2401, 0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401,
    0x3001, 0x2801, 0x2401, 0x2201, 0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101,
    0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1, 0x0221, 0x0141, 0x0111, 0x0085,
    0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
__constant__ uint8_t c_nmps[47] = {
    1, 2, 3, 4, 5, 38, 7, 8, 9, 10, 11, 12, 13, 29, 15, 16, 17, 18, 19, 20,
    21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40,
    41, 42, 43, 44, 45, 45, 46};
__constant__ uint8_t c_nlps[47] = {
    1, 6, 9, 12, 29, 33, 6, 14, 14, 14, 17, 18, 20, 21, 14, 14, 15, 16, 17, 18,
    19, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37,
    38, 39, 40, 41, 42, 43, 46};

struct Tables {
    uint32_t mq[48];          // packed states: Qe << 16 | NMPS << 1 | NLPS << 7 | SWITCH << 13 (bit 0: MPS)
    uint8_t zc[4][512];       // zero-coding label per orientation and 3x3 neighbourhood
    uint8_t sc[256];          // sign label | XOR bit << 4
    // Decoder context words by 2 * state + MPS: Qe << 16, the entry after an
    // LPS << 7 (NLPS, MPS switched where SWITCH is set), the entry after an
    // MPS (NMPS, same MPS) in bits 0-6, whose bit 0 is the MPS.
    uint32_t mqd[96];
};

// Zero-coding label from neighbour counts, ISO Table D.1 (the reference's
// SPCXLUT, coefficient_coder.cl:330-393).
__device__ int zc_label(int orient, int h, int v, int d)
{
    if (orient == 1) { const int t = h; h = v; v = t; }
    if (orient == 3) {
        const int hv = h + v;
        if (d >= 3) return 8;
        if (d == 2) return hv >= 1 ? 7 : 6;
        if (d == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
        return hv >= 2 ? 2 : hv;
    }
    if (h == 2) return 8;
    if (h == 1) return v >= 1 ? 7 : (d >= 1 ? 6 : 5);
    if (v == 2) return 4;
    if (v == 1) return 3;
    return d >= 2 ? 2 : d;
}

__device__ void build_tables(Tables &t)
{
    for (int i = threadIdx.x; i < 47; i += blockDim.x)
        t.mq[i] = ((uint32_t)c_qe[i] << 16) | ((uint32_t)c_nmps[i] << 1) | ((uint32_t)c_nlps[i] << 7) |
                  ((uint32_t)(i == 0 || i == 6 || i == 14) << 13);
    for (int i = threadIdx.x; i < 94; i += blockDim.x) {
        const int st = i >> 1, mps = i & 1, sw = st == 0 || st == 6 || st == 14;
        t.mqd[i] = ((uint32_t)c_qe[st] << 16) | ((uint32_t)(2 * c_nlps[st] + (mps ^ sw)) << 7) |
                   (uint32_t)(2 * c_nmps[st] + mps);
    }
    // 3x3 neighbourhood bits: 0 up-left 1 up 2 up-right 3 left 4 self
    // 5 right 6 down-left 7 down 8 down-right.
    for (int i = threadIdx.x; i < 4 * 512; i += blockDim.x) {
        const int o = i >> 9, p = i & 511;
        const int h = ((p >> 3) & 1) + ((p >> 5) & 1);
        const int v = ((p >> 1) & 1) + ((p >> 7) & 1);
        const int d = (p & 1) + ((p >> 2) & 1) + ((p >> 6) & 1) + ((p >> 8) & 1);
        t.zc[o][p] = (uint8_t)zc_label(o, h, v, d);
    }
    // Sign index: neighbourhood bits 1,3,5,7 (significance of up, left,
    // right, down) with the neighbours' signs one bit below them.
    // ISO Tables D.2/D.3 (signcxlut, coefficient_coder.cl:406-435).
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        auto ctb = [&](int sig, int neg) { return sig ? (neg ? -1 : 1) : 0; };
        int vc = ctb((i >> 1) & 1, i & 1) + ctb((i >> 7) & 1, (i >> 6) & 1);
        int hc = ctb((i >> 3) & 1, (i >> 2) & 1) + ctb((i >> 5) & 1, (i >> 4) & 1);
        hc = hc > 1 ? 1 : (hc < -1 ? -1 : hc);
        vc = vc > 1 ? 1 : (vc < -1 ? -1 : vc);
        int cx, xr;
        if (hc == 0) {
            cx = vc == 0 ? 9 : 10;
            xr = vc < 0;
        } else {
            cx = 12 + hc * vc;
            xr = hc < 0;
        }
        t.sc[i] = (uint8_t)(cx | (xr << 4));
    }
}

// Sign-coding index of row y (= 4s+k) of column c from the flag word's
// 3x3 neighbourhood n9 and the sign words of columns c-1, c, c+1 (sgn has a
// zero guard column on each side: column c is sgn[c + 1]).
__device__ __forceinline__ uint32_t sign_index(const unsigned long long *sgn, uint32_t n9, int c, int y)
{
    const unsigned long long sl = sgn[c], sc = sgn[c + 1], sr = sgn[c + 2];
    const uint32_t up = y > 0 ? (uint32_t)(sc >> (y - 1)) & 1u : 0u;
    const uint32_t dn = y < 63 ? (uint32_t)(sc >> (y + 1)) & 1u : 0u;
    const uint32_t lf = (uint32_t)(sl >> y) & 1u, rt = (uint32_t)(sr >> y) & 1u;
    return (n9 & 0xAAu) | up | (lf << 2) | (rt << 4) | (dn << 6);
}

// Record that row k of stripe s in column c became significant: the flag
// words of the neighbouring columns and of the stripes above and below see
// it through their neighbourhood bits.  With vertically causal contexts
// (vsc, ISO D.7) the stripe above does not: its last row's neighbourhood
// then leaves out the row below for every context (zero coding, sign, run
// mode, refinement).
__device__ __forceinline__ void mark_significant(uint32_t *F, unsigned long long *sgn, int s, int k, int c, int w,
                                                 int nstripes, uint32_t neg, bool vsc = false)
{
    const int i = s * 64 + c;
    if (c > 0) F[i - 1] |= 1u << (3 * k + 5);
    if (c + 1 < w) F[i + 1] |= 1u << (3 * k + 3);
    if (k == 0 && s > 0 && !vsc) {
        const int u = i - 64;
        F[u] |= 1u << 16;
        if (c > 0) F[u - 1] |= 1u << 17;
        if (c + 1 < w) F[u + 1] |= 1u << 15;
    }
    if (k == 3 && s + 1 < nstripes) {
        const int d = i + 64;
        F[d] |= 1u << 1;
        if (c > 0) F[d - 1] |= 1u << 2;
        if (c + 1 < w) F[d + 1] |= 1u << 0;
    }
    if (neg) sgn[c + 1] |= 1ull << (4 * s + k);
}

// Code-block style (ISO Table A.19): whether coding pass t (0: the first
// cleanup pass) ends a codeword segment (D.4.2, D.6), whether it is raw-coded
// (bypass: SPP and MRP from the 11th pass on), and the segments that passes
// [0, passes) span.
__host__ __device__ __forceinline__ bool style_pass_terminates(int style, int t)
{
    if (style & TC_CBLK_STYLE_TERMALL) return true;
    if (style & TC_CBLK_STYLE_BYPASS) return t == 9 || (t >= 10 && t % 3 != 1);
    return false;
}
__host__ __device__ __forceinline__ bool style_pass_raw(int style, int t)
{
    return (style & TC_CBLK_STYLE_BYPASS) && t >= 10 && t % 3 != 0;
}
__host__ __device__ __forceinline__ int style_segments(int style, int passes)
{
    int n = passes > 0;
    for (int t = 0; t + 1 < passes; t++) n += style_pass_terminates(style, t);
    return n;
}
// Candidate mask of the group's columns: column gl + G*j for predicate any[j].
template <int G>
__device__ __forceinline__ unsigned long long group_ballot(const bool (&any)[64 / G], unsigned gmask, int gshift)
{
    unsigned long long m = 0;
#pragma unroll
    for (int j = 0; j < 64 / G; j++) {
        const unsigned b = __ballot_sync(gmask, any[j]);
        m |= (unsigned long long)((G == 32 ? b : (b >> gshift)) & (G == 32 ? 0xffffffffu : ((1u << G) - 1u))) << (G * j);
    }
    return m;
}

}  // namespace
}  // namespace tc
