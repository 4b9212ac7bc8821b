// t1_decode.cu -- Tier-1 EBCOT/MQ code-block decoder for sm_100a.
//
// Replaces the reference g_decode kernel (coefficient_coder.cl:778-819) and
// the dequantiser kernels (quantizer_*_inverse.cl) with one persistent
// launch:
//   * one warp per code-block; warps pull block indices from a device work
//     queue (an atomic counter over a longest-first order), so blocks of
//     uneven size and pass count from many tiles and images share a launch;
//   * the code-block state lives in shared memory as one 64-bit word per
//     column and per state bit (significance, sign, refined, visited), so
//     the 3x6 neighbourhood of a stripe column is three 6-bit windows and a
//     context label is one table lookup (the reference rebuilds a 3x3 window
//     of packed words from global memory at every step, :271-298);
//   * the MQ interval state (A, C, CT, byte position) stays in registers and
//     each context's probability state is one packed word, so the common MPS
//     path of a decision is a shared load, two compares and a subtract;
//   * the pass loop honours the coding-pass count (defect D3 fixed) and
//     updates the state it reads (defects D1/D2 fixed);
//   * the warp's lanes clear the state, and write the block out coalesced
//     with the inverse quantiser fused in (ISO E.1, reconstruction point r).
#include <cuda_runtime.h>

#include <algorithm>

#include "tc_internal.cuh"

namespace tc {
namespace {

constexpr int kWarps = 4;         // warps (code-blocks in flight) per CTA
constexpr int kCols = 66;         // 64 columns + a zero column on each side

// ISO Table C.2 (coefficient_coder.cl:36-60), packed per state index as
// Qe | NMPS << 16 | NLPS << 22 | SWITCH << 28.
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

template <typename MagT>
struct WarpState {
    unsigned long long sig[kCols];   // significance, bit r = row r
    unsigned long long sgn[kCols];   // sign (1 = negative)
    unsigned long long ref[kCols];   // refined at least once (sigma')
    unsigned long long vis[kCols];   // coded in this plane's significance pass (pi)
    uint32_t ctx[20];                // packed probability state per context
    uint8_t mrow[64];                // refinement pass: rows of the stripe to refine
    uint8_t mctx[64];                // refinement pass: 2-bit context code per row
    MagT mag[64 * 64];               // magnitude bits decoded so far
};

struct Tables {
    uint32_t mq[48];          // packed probability states
    uint8_t zc[4][256];       // zero-coding label per orientation and 8-neighbour pattern
    uint8_t sc[256];          // sign label | XOR bit << 4
};

// Zero-coding label from neighbour counts, ISO Table D.1 (the reference's
// SPCXLUT, coefficient_coder.cl:330-393, indexes the same table by a 9-bit
// window; here the index is an 8-bit neighbour pattern).
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
        t.mq[i] = (uint32_t)c_qe[i] | ((uint32_t)c_nmps[i] << 16) | ((uint32_t)c_nlps[i] << 22) |
                  ((uint32_t)(i == 0 || i == 6 || i == 14) << 28);
    // Pattern bits: 0-2 left column rows k-1..k+1, 3 centre row k-1,
    // 4 centre row k+1, 5-7 right column rows k-1..k+1.
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) {
        const int o = i >> 8, p = i & 255;
        const int h = ((p >> 1) & 1) + ((p >> 6) & 1);
        const int v = ((p >> 3) & 1) + ((p >> 4) & 1);
        const int d = (p & 1) + ((p >> 2) & 1) + ((p >> 5) & 1) + ((p >> 7) & 1);
        t.zc[o][p] = (uint8_t)zc_label(o, h, v, d);
    }
    // Sign index bits: 0 sigL 1 sgnL 2 sigR 3 sgnR 4 sigU 5 sgnU 6 sigD 7 sgnD.
    // ISO Tables D.2/D.3 (signcxlut, coefficient_coder.cl:406-435).
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        auto ctb = [&](int s, int n) { return s ? (n ? -1 : 1) : 0; };
        int hc = ctb(i & 1, (i >> 1) & 1) + ctb((i >> 2) & 1, (i >> 3) & 1);
        int vc = ctb((i >> 4) & 1, (i >> 5) & 1) + ctb((i >> 6) & 1, (i >> 7) & 1);
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

// MQ decoder (ISO C.3; bytein/renormd/mqDecode, coefficient_coder.cl:121-252).
struct MQ {
    const uint8_t *p;
    int len, bp, ct;
    uint32_t a, c;

    __device__ __forceinline__ uint32_t byte_at(int i) const { return i < len ? (uint32_t)__ldg(p + i) : 0xFFu; }
    __device__ __forceinline__ void bytein()
    {
        const uint32_t b = byte_at(bp);
        if (b == 0xFF) {
            const uint32_t b1 = byte_at(bp + 1);
            if (b1 > 0x8F) {
                c += 0xFF00;
                ct = 8;
            } else {
                bp++;
                c += b1 << 9;
                ct = 7;
            }
        } else {
            bp++;
            c += byte_at(bp) << 8;
            ct = 8;
        }
        // keep the codeword stream ahead of the decoder in L1
        if ((bp & 63) == 0 && bp + 256 < len) asm volatile("prefetch.global.L1 [%0];" ::"l"(p + bp + 256));
    }
    __device__ __forceinline__ void init(const uint8_t *d, int n)
    {
        p = d;
        len = n;
        bp = 0;
        c = byte_at(0) << 16;
        bytein();
        c <<= 7;
        ct -= 7;
        a = 0x8000;
    }
    __device__ __forceinline__ void renorm()
    {
        int sh = __clz(a) - 16;
        while (sh > 0) {
            if (ct == 0) bytein();
            const int s = sh < ct ? sh : ct;
            a <<= s;
            c <<= s;
            ct -= s;
            sh -= s;
        }
    }
    __device__ __forceinline__ int decode(uint32_t *ctx, const uint32_t *tbl, int cx)
    {
        const uint32_t w = ctx[cx];
        const uint32_t qe = w & 0xFFFF, mps = w >> 31;
        a -= qe;
        if ((c >> 16) < qe) {
            uint32_t d;
            if (a < qe) {
                d = mps;
                ctx[cx] = tbl[(w >> 16) & 63] | (mps << 31);
            } else {
                d = mps ^ 1;
                ctx[cx] = tbl[(w >> 22) & 63] | ((mps ^ ((w >> 28) & 1)) << 31);
            }
            a = qe;
            renorm();
            return (int)d;
        }
        c -= qe << 16;
        if (a & 0x8000) return (int)mps;
        uint32_t d;
        if (a < qe) {
            d = mps ^ 1;
            ctx[cx] = tbl[(w >> 22) & 63] | ((mps ^ ((w >> 28) & 1)) << 31);
        } else {
            d = mps;
            ctx[cx] = tbl[(w >> 16) & 63] | (mps << 31);
        }
        renorm();
        return (int)d;
    }
};

// Rows 4s-1 .. 4s+4 of a column word as a 6-bit window.
__device__ __forceinline__ uint32_t win6(unsigned long long w, int s)
{
    return s == 0 ? (uint32_t)((w << 1) & 0x3Full) : (uint32_t)((w >> (4 * s - 1)) & 0x3Full);
}

__device__ __forceinline__ uint32_t zc_pattern(uint32_t wl, uint32_t wc, uint32_t wr, int k)
{
    const uint32_t cc = (wc >> k) & 5u;
    return ((wl >> k) & 7u) | (((cc & 1u) | ((cc >> 1) & 2u)) << 3) | (((wr >> k) & 7u) << 5);
}

__device__ __forceinline__ uint32_t sc_index(uint32_t wl, uint32_t sl, uint32_t wc, uint32_t sc,
                                             uint32_t wr, uint32_t sr, int k)
{
    return ((wl >> (k + 1)) & 1u) | (((sl >> (k + 1)) & 1u) << 1) | (((wr >> (k + 1)) & 1u) << 2) |
           (((sr >> (k + 1)) & 1u) << 3) | (((wc >> k) & 1u) << 4) | (((sc >> k) & 1u) << 5) |
           (((wc >> (k + 2)) & 1u) << 6) | (((sc >> (k + 2)) & 1u) << 7);
}

// Rows of a stripe in which a coefficient has at least one significant
// neighbour (bit k = row 4s+k).
__device__ __forceinline__ uint32_t nb_rows(uint32_t wl, uint32_t wc, uint32_t wr)
{
    const uint32_t n = wl | wr;
    return ((n | (n >> 1) | (n >> 2)) | (wc | (wc >> 2))) & 0xFu;
}

// Lane-parallel candidate test for the significance pass: does column c
// (window rows of stripe s) hold an insignificant coefficient with a
// significant neighbour?
template <typename MagT>
__device__ __forceinline__ bool spp_candidate(const WarpState<MagT> &S, int c, int s, uint32_t rmask)
{
    const uint32_t wl = win6(S.sig[c], s), wc = win6(S.sig[c + 1], s), wr = win6(S.sig[c + 2], s);
    return (~(wc >> 1) & rmask & nb_rows(wl, wc, wr)) != 0u;
}

// Decode one code-block.  Every lane of the warp runs this function in
// lock-step (the MQ state is replicated, shared-memory accesses are
// broadcasts); lanes split the per-stripe candidate searches between them
// (lane l owns columns l and l+32) and the serial loop visits only the
// candidate columns, in scan order.  Returns the last pass type (0 cleanup,
// 1 significance propagation, 2 refinement) and its plane.
template <typename MagT>
__device__ int decode_block(WarpState<MagT> &S, const Tables &T, const uint8_t *seg, int len, int w,
                            int h, int orient, int numbps, int passes, int *last_plane, int lane)
{
    MQ mq;
    mq.init(seg, len);
    uint32_t *ctx = S.ctx;
    const uint32_t *tbl = T.mq;
    const uint8_t *zc = T.zc[orient];
    const int nstripes = (h + 3) >> 2;
    const int c0 = lane, c1 = lane + 32;
    int type = 0, pass = 0;
    *last_plane = numbps - 1;

    for (int p = numbps - 1; p >= 0; --p) {
        const MagT pbit = (MagT)(1u << p);
        if (p != numbps - 1) {
            // ---- significance propagation pass (ISO D.3.1; SigPropPassFunctor) ----
            for (int s = 0; s < nstripes; s++) {
                const int rows = min(4, h - 4 * s);
                const uint32_t rmask = (1u << rows) - 1u;
                __syncwarp();
                const bool a0 = c0 < w && spp_candidate(S, c0, s, rmask);
                const bool a1 = c1 < w && spp_candidate(S, c1, s, rmask);
                unsigned long long cand = (unsigned long long)__ballot_sync(0xffffffffu, a0) |
                                          ((unsigned long long)__ballot_sync(0xffffffffu, a1) << 32);
                while (cand) {
                    const int c = __ffsll((long long)cand) - 1;
                    cand &= cand - 1;
                    const uint32_t wl = win6(S.sig[c], s), wr = win6(S.sig[c + 2], s);
                    uint32_t wc = win6(S.sig[c + 1], s);
                    const uint32_t wc0 = wc;
                    uint32_t sc = win6(S.sgn[c + 1], s);
                    uint32_t vmask = 0;
                    for (int k = 0; k < rows; k++) {
                        if ((wc >> (k + 1)) & 1u) continue;
                        const uint32_t pat = zc_pattern(wl, wc, wr, k);
                        if (!pat) continue;
                        vmask |= 1u << k;
                        if (mq.decode(ctx, tbl, zc[pat])) {
                            const uint32_t sl = win6(S.sgn[c], s), sr = win6(S.sgn[c + 2], s);
                            const uint32_t si = T.sc[sc_index(wl, sl, wc, sc, wr, sr, k)];
                            const uint32_t neg = (uint32_t)mq.decode(ctx, tbl, si & 15) ^ (si >> 4);
                            wc |= 2u << k;
                            sc |= neg << (k + 1);
                            S.mag[(4 * s + k) * 64 + c] = pbit;
                        }
                    }
                    if (wc != wc0) {
                        S.sig[c + 1] |= (unsigned long long)((wc >> 1) & 0xFu) << (4 * s);
                        S.sgn[c + 1] |= (unsigned long long)((sc >> 1) & 0xFu) << (4 * s);
                        if (c + 1 < w) cand |= 1ull << (c + 1);  // the next column gained a neighbour
                    }
                    if (vmask) S.vis[c + 1] |= (unsigned long long)vmask << (4 * s);
                }
            }
            type = 1;
            *last_plane = p;
            if (++pass >= passes) break;
            __syncwarp();

            // ---- magnitude refinement pass (ISO D.3.3; MagRefPassFunctor) ----
            // The rows to refine and their contexts do not change during the
            // pass, so the lanes precompute them for their columns.
            for (int s = 0; s < nstripes; s++) {
                const int rows = min(4, h - 4 * s);
                const uint32_t rmask = (1u << rows) - 1u;
                bool any[2];
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int c = lane + 32 * j;
                    uint32_t rr = 0, codes = 0;
                    if (c < w) {
                        const uint32_t wl = win6(S.sig[c], s), wc = win6(S.sig[c + 1], s),
                                       wr = win6(S.sig[c + 2], s);
                        const uint32_t vis = (uint32_t)(S.vis[c + 1] >> (4 * s)) & 0xFu;
                        const uint32_t ref = (uint32_t)(S.ref[c + 1] >> (4 * s)) & 0xFu;
                        rr = (wc >> 1) & rmask & ~vis;
                        for (int k = 0; k < 4; k++)
                            codes |= (((ref >> k) & 1u) ? 2u : (zc_pattern(wl, wc, wr, k) ? 1u : 0u)) << (2 * k);
                        S.mrow[c] = (uint8_t)rr;
                        S.mctx[c] = (uint8_t)codes;
                        S.ref[c + 1] |= (unsigned long long)rr << (4 * s);
                    }
                    any[j] = rr != 0;
                }
                unsigned long long cand = (unsigned long long)__ballot_sync(0xffffffffu, any[0]) |
                                          ((unsigned long long)__ballot_sync(0xffffffffu, any[1]) << 32);
                __syncwarp();
                while (cand) {
                    const int c = __ffsll((long long)cand) - 1;
                    cand &= cand - 1;
                    uint32_t rr = S.mrow[c];
                    const uint32_t codes = S.mctx[c];
                    while (rr) {
                        const int k = __ffs(rr) - 1;
                        rr &= rr - 1;
                        if (mq.decode(ctx, tbl, 14 + ((codes >> (2 * k)) & 3u))) S.mag[(4 * s + k) * 64 + c] |= pbit;
                    }
                }
                __syncwarp();
            }
            type = 2;
            if (++pass >= passes) break;
        }

        // ---- cleanup pass (ISO D.3.4; CleanUpPassFunctor) ----
        for (int s = 0; s < nstripes; s++) {
            const int rows = min(4, h - 4 * s);
            const uint32_t rmask = (1u << rows) - 1u;
            __syncwarp();
            bool any[2];
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int c = lane + 32 * j;
                any[j] = c < w && ((~(uint32_t)((S.sig[c + 1] | S.vis[c + 1]) >> (4 * s))) & rmask) != 0u;
            }
            unsigned long long cand = (unsigned long long)__ballot_sync(0xffffffffu, any[0]) |
                                      ((unsigned long long)__ballot_sync(0xffffffffu, any[1]) << 32);
            while (cand) {
                const int c = __ffsll((long long)cand) - 1;
                cand &= cand - 1;
                const uint32_t wl = win6(S.sig[c], s), wr = win6(S.sig[c + 2], s);
                uint32_t wc = win6(S.sig[c + 1], s);
                const uint32_t wc0 = wc;
                const uint32_t vis = (uint32_t)(S.vis[c + 1] >> (4 * s)) & 0xFu;
                uint32_t sc = win6(S.sgn[c + 1], s);
                int k = 0;
                if (rows == 4 && (wl | wc | wr) == 0u) {
                    // run-length mode: four rows with an all-zero neighbourhood
                    if (!mq.decode(ctx, tbl, 18)) continue;
                    int r = mq.decode(ctx, tbl, 17) << 1;
                    r |= mq.decode(ctx, tbl, 17);
                    const uint32_t sl = win6(S.sgn[c], s), sr = win6(S.sgn[c + 2], s);
                    const uint32_t si = T.sc[sc_index(wl, sl, wc, sc, wr, sr, r)];
                    const uint32_t neg = (uint32_t)mq.decode(ctx, tbl, si & 15) ^ (si >> 4);
                    wc |= 2u << r;
                    sc |= neg << (r + 1);
                    S.mag[(4 * s + r) * 64 + c] = pbit;
                    k = r + 1;
                }
                for (; k < rows; k++) {
                    if (((wc >> (k + 1)) | (vis >> k)) & 1u) continue;
                    if (mq.decode(ctx, tbl, zc[zc_pattern(wl, wc, wr, k)])) {
                        const uint32_t sl = win6(S.sgn[c], s), sr = win6(S.sgn[c + 2], s);
                        const uint32_t si = T.sc[sc_index(wl, sl, wc, sc, wr, sr, k)];
                        const uint32_t neg = (uint32_t)mq.decode(ctx, tbl, si & 15) ^ (si >> 4);
                        wc |= 2u << k;
                        sc |= neg << (k + 1);
                        S.mag[(4 * s + k) * 64 + c] = pbit;
                    }
                }
                if (wc != wc0) {
                    S.sig[c + 1] |= (unsigned long long)((wc >> 1) & 0xFu) << (4 * s);
                    S.sgn[c + 1] |= (unsigned long long)((sc >> 1) & 0xFu) << (4 * s);
                }
            }
        }
        type = 0;
        *last_plane = p;
        if (++pass >= passes) break;
        __syncwarp();
        for (int c = lane; c < kCols; c += 32) S.vis[c] = 0ull;
        __syncwarp();
    }
    return type;
}

template <typename MagT>
__global__ void __launch_bounds__(32 * kWarps)
t1_decode_kernel(const tc_cblk_desc *__restrict__ desc, const uint32_t *__restrict__ order, int n, int ndesc,
                 const uint8_t *__restrict__ pool, uint64_t pool_len, char *__restrict__ out, int out_mode,
                 float recon_r, uint32_t *__restrict__ counter, uint32_t *__restrict__ err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    Tables &T = *reinterpret_cast<Tables *>(smem);
    WarpState<MagT> *states =
        reinterpret_cast<WarpState<MagT> *>(smem + ((sizeof(Tables) + 15) & ~size_t(15)));
    build_tables(T);
    __syncthreads();

    const int lane = threadIdx.x & 31;
    WarpState<MagT> &S = states[threadIdx.x >> 5];

    for (;;) {
        int idx = 0;
        if (lane == 0) idx = (int)atomicAdd(counter, 1u);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= n) break;
        const uint32_t bi = order ? order[idx] : (uint32_t)idx;
        if (bi >= (uint32_t)ndesc) {
            if (lane == 0) atomicOr(err, TC_DERR_DESC);
            continue;
        }
        const tc_cblk_desc d = desc[bi];
        const int w = d.w, h = d.h;
        const bool geom_ok = w >= 1 && w <= 64 && h >= 1 && h <= 64;
        const int numbps = (int)d.mb - (int)d.zero_bitplanes;
        bool ok = geom_ok && d.mb >= 1 && d.mb <= 31 && d.orient <= 3 && numbps >= 0 &&
                  (numbps == 0 || d.passes <= 3 * numbps - 2) && numbps <= (int)(8 * sizeof(MagT));
        const bool pool_ok = d.seg_off <= pool_len && (uint64_t)d.seg_len <= pool_len - d.seg_off;
        if (!geom_ok) {
            if (lane == 0) atomicOr(err, TC_DERR_DESC);
            continue;
        }
        if (!ok || !pool_ok) {
            if (lane == 0) atomicOr(err, ok ? TC_DERR_POOL : TC_DERR_DESC);
            ok = false;
        }
        const bool coded = ok && numbps > 0 && d.passes > 0;

        // clear the column state words (all lanes)
        for (int i = lane; i < kCols; i += 32) {
            S.sig[i] = 0ull;
            S.sgn[i] = 0ull;
            S.ref[i] = 0ull;
            S.vis[i] = 0ull;
        }
        if (lane < 19) {
            const int st = lane == 0 ? 4 : (lane == 17 ? 46 : (lane == 18 ? 3 : 0));
            S.ctx[lane] = T.mq[st];
        }
        __syncwarp();

        int type = 0, last_plane = 0;
        if (coded)
            type = decode_block(S, T, pool + d.seg_off, (int)d.seg_len, w, h, d.orient, numbps, d.passes,
                                &last_plane, lane);
        __syncwarp();

        // epilogue: reconstruction + inverse quantisation, coalesced rows
        const bool irrev = (d.flags & TC_CBLK_IRREVERSIBLE) != 0;
        const float half_step = recon_r;
        for (int y = 0; y < h; y++) {
            char *row = out + 4 * (d.out_off + (uint64_t)y * d.out_pitch);
            for (int x = lane; x < w; x += 32) {
                const bool sg = coded && ((S.sig[x + 1] >> y) & 1ull);
                uint32_t mg = 0, neg = 0, u = 0;
                if (sg) {
                    mg = (uint32_t)S.mag[y * 64 + x];
                    neg = (uint32_t)(S.sgn[x + 1] >> y) & 1u;
                    u = (uint32_t)last_plane;
                    if (type == 1 && !((S.vis[x + 1] >> y) & 1ull)) u++;
                }
                if (out_mode == TC_T1_OUT_RAW) {
                    reinterpret_cast<uint32_t *>(row)[x] = sg ? ((mg << (31 - d.mb)) | (neg << 31)) : 0u;
                } else if (irrev) {
                    float v = 0.0f;
                    if (sg) v = ((float)mg + half_step * (float)(1u << u)) * d.step;
                    reinterpret_cast<float *>(row)[x] = neg ? -v : v;
                } else {
                    int32_t v = 0;
                    if (sg) v = (int32_t)mg + (u ? (int32_t)floorf(half_step * (float)(1u << u)) : 0);
                    reinterpret_cast<int32_t *>(row)[x] = neg ? -v : v;
                }
            }
        }
        __syncwarp();
    }
}

// Standalone inverse quantiser over raw sign-magnitude words.
__global__ void dequant_raw_kernel(const tc_cblk_desc *__restrict__ desc, int n,
                                   const uint32_t *__restrict__ raw, char *__restrict__ out,
                                   float recon_r, uint32_t *words)
{
    const int b = blockIdx.x;
    if (b >= n) return;
    const tc_cblk_desc d = desc[b];
    if (d.w < 1 || d.w > 64 || d.h < 1 || d.h > 64 || d.mb < 1 || d.mb > 31) {
        if (threadIdx.x == 0) atomicOr(&words[0], TC_DERR_DESC);
        return;
    }
    const int numbps = (int)d.mb - (int)d.zero_bitplanes;
    // Decoded planes from the pass count: the last pass ran on plane p_last.
    int u = 0;
    if (numbps > 0 && d.passes > 0) {
        const int p_last = numbps - 1 - (d.passes + 1) / 3;
        u = p_last < 0 ? 0 : p_last;
    }
    const bool irrev = (d.flags & TC_CBLK_IRREVERSIBLE) != 0;
    for (int i = threadIdx.x; i < d.w * d.h; i += blockDim.x) {
        const int y = i / d.w, x = i - y * d.w;
        const uint64_t o = d.out_off + (uint64_t)y * d.out_pitch + x;
        const uint32_t r = raw[o];
        const uint32_t mg = (r & 0x7FFFFFFFu) >> (31 - d.mb);
        const bool neg = (r >> 31) != 0;
        if (irrev) {
            float v = mg ? ((float)mg + recon_r * (float)(1u << u)) * d.step : 0.0f;
            reinterpret_cast<float *>(out)[o] = neg ? -v : v;
        } else {
            int32_t v = mg ? (int32_t)mg + (u ? (int32_t)floorf(recon_r * (float)(1u << u)) : 0) : 0;
            reinterpret_cast<int32_t *>(out)[o] = neg ? -v : v;
        }
    }
}

}  // namespace

namespace {
template <typename MagT>
cudaError_t launch_class(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order, int n, int ndesc,
                         const uint8_t *d_pool, uint64_t pool_len, void *d_out, int out_mode, float recon_r,
                         int slot)
{
    const size_t smem = ((sizeof(Tables) + 15) & ~size_t(15)) + kWarps * sizeof(WarpState<MagT>);
    cudaError_t e = cudaFuncSetAttribute(t1_decode_kernel<MagT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, t1_decode_kernel<MagT>, 32 * kWarps, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const int want = (n + kWarps - 1) / kWarps;
    const int grid = std::min(want, per_sm * num_sms(ctx->device));
    e = cudaMemsetAsync(ctx->d_words + slot, 0, sizeof(uint32_t), ctx->stream);
    if (e != cudaSuccess) return e;
    t1_decode_kernel<MagT><<<grid, 32 * kWarps, smem, ctx->stream>>>(
        d_desc, d_order, n, ndesc, d_pool, pool_len, static_cast<char *>(d_out), out_mode, recon_r,
        ctx->d_words + slot, ctx->d_words);
    ctx->launches++;
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_t1_decode(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order, int n,
                             const uint8_t *d_pool, uint64_t pool_len, void *d_out, int out_mode, float recon_r,
                             int max_bitplanes)
{
    return launch_t1_classes(ctx, d_desc, d_order, n, max_bitplanes <= 8 ? n : 0,
                             max_bitplanes > 8 && max_bitplanes <= 16 ? n : 0, max_bitplanes > 16 ? n : 0, d_pool,
                             pool_len, d_out, out_mode, recon_r);
}

cudaError_t launch_t1_classes(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order, int ndesc,
                              int n8, int n16, int n32, const uint8_t *d_pool, uint64_t pool_len, void *d_out,
                              int out_mode, float recon_r)
{
    cudaError_t e = cudaSuccess;
    if (n8 > 0)
        e = launch_class<uint8_t>(ctx, d_desc, d_order, n8, ndesc, d_pool, pool_len, d_out, out_mode, recon_r, 1);
    if (e == cudaSuccess && n16 > 0)
        e = launch_class<uint16_t>(ctx, d_desc, d_order ? d_order + n8 : nullptr, n16, ndesc, d_pool, pool_len,
                                   d_out, out_mode, recon_r, 2);
    if (e == cudaSuccess && n32 > 0)
        e = launch_class<uint32_t>(ctx, d_desc, d_order ? d_order + n8 + n16 : nullptr, n32, ndesc, d_pool,
                                   pool_len, d_out, out_mode, recon_r, 3);
    return e;
}

cudaError_t launch_dequant_raw(tc_ctx *ctx, const tc_cblk_desc *d_desc, int n, const uint32_t *d_raw,
                               void *d_out, float recon_r)
{
    if (n <= 0) return cudaSuccess;
    dequant_raw_kernel<<<n, 256, 0, ctx->stream>>>(d_desc, n, d_raw, static_cast<char *>(d_out), recon_r,
                                                   ctx->d_words);
    ctx->launches++;
    return cudaGetLastError();
}

}  // namespace tc
