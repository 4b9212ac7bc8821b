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

struct WarpState {
    unsigned long long sig[kCols];
    unsigned long long sgn[kCols];
    unsigned long long ref[kCols];
    unsigned long long vis[kCols];
    uint32_t ctx[20];
    uint32_t mag[64 * 64];
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

// Serial decode of one code-block by one lane.  Returns the last pass type
// (0 cleanup, 1 significance propagation, 2 refinement) and its plane.
__device__ int decode_block(WarpState &S, const Tables &T, const uint8_t *seg, int len, int w,
                            int h, int orient, int numbps, int passes, int *last_plane)
{
    MQ mq;
    mq.init(seg, len);
    uint32_t *ctx = S.ctx;
    const uint32_t *tbl = T.mq;
    const uint8_t *zc = T.zc[orient];
    const int nstripes = (h + 3) >> 2;
    int type = 0, pass = 0;
    *last_plane = numbps - 1;

    for (int p = numbps - 1; p >= 0; --p) {
        const uint32_t pbit = 1u << p;
        if (p != numbps - 1) {
            // ---- significance propagation pass (ISO D.3.1; SigPropPassFunctor) ----
            for (int s = 0; s < nstripes; s++) {
                const int rows = min(4, h - 4 * s);
                const uint32_t rmask = (1u << rows) - 1u;
                uint32_t wl = 0, sl = 0;
                uint32_t wc = win6(S.sig[1], s), sc = win6(S.sgn[1], s);
                for (int c = 0; c < w; c++) {
                    const uint32_t wr = win6(S.sig[c + 2], s), sr = win6(S.sgn[c + 2], s);
                    const uint32_t insig = ~(wc >> 1) & rmask;
                    if (insig & nb_rows(wl, wc, wr)) {
                        uint32_t vmask = 0;
                        const uint32_t wc0 = wc;
                        for (int k = 0; k < rows; k++) {
                            if ((wc >> (k + 1)) & 1u) continue;
                            const uint32_t pat = zc_pattern(wl, wc, wr, k);
                            if (!pat) continue;
                            vmask |= 1u << k;
                            if (mq.decode(ctx, tbl, zc[pat])) {
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
                        S.vis[c + 1] |= (unsigned long long)vmask << (4 * s);
                    }
                    wl = wc;
                    sl = sc;
                    wc = wr;
                    sc = sr;
                }
            }
            type = 1;
            *last_plane = p;
            if (++pass >= passes) break;

            // ---- magnitude refinement pass (ISO D.3.3; MagRefPassFunctor) ----
            for (int s = 0; s < nstripes; s++) {
                const int rows = min(4, h - 4 * s);
                const uint32_t rmask = (1u << rows) - 1u;
                uint32_t wl = 0, wc = win6(S.sig[1], s);
                for (int c = 0; c < w; c++) {
                    const uint32_t wr = win6(S.sig[c + 2], s);
                    const uint32_t vis = (uint32_t)(S.vis[c + 1] >> (4 * s)) & 0xFu;
                    const uint32_t cand = (wc >> 1) & rmask & ~vis;
                    if (cand) {
                        const uint32_t ref = (uint32_t)(S.ref[c + 1] >> (4 * s)) & 0xFu;
                        for (int k = 0; k < rows; k++) {
                            if (!((cand >> k) & 1u)) continue;
                            const int cx = ((ref >> k) & 1u) ? 16 : (zc_pattern(wl, wc, wr, k) ? 15 : 14);
                            if (mq.decode(ctx, tbl, cx)) S.mag[(4 * s + k) * 64 + c] |= pbit;
                        }
                        S.ref[c + 1] |= (unsigned long long)cand << (4 * s);
                    }
                    wl = wc;
                    wc = wr;
                }
            }
            type = 2;
            if (++pass >= passes) break;
        }

        // ---- cleanup pass (ISO D.3.4; CleanUpPassFunctor) ----
        for (int s = 0; s < nstripes; s++) {
            const int rows = min(4, h - 4 * s);
            uint32_t wl = 0, sl = 0;
            uint32_t wc = win6(S.sig[1], s), sc = win6(S.sgn[1], s);
            for (int c = 0; c < w; c++) {
                const uint32_t wr = win6(S.sig[c + 2], s), sr = win6(S.sgn[c + 2], s);
                const uint32_t vis = (uint32_t)(S.vis[c + 1] >> (4 * s)) & 0xFu;
                const uint32_t wc0 = wc;
                int k = 0;
                bool run_done = false;
                if (rows == 4 && (wl | wc | wr) == 0u) {
                    // run-length mode: four rows with an all-zero neighbourhood
                    if (!mq.decode(ctx, tbl, 18)) {
                        run_done = true;
                    } else {
                        int r = mq.decode(ctx, tbl, 17) << 1;
                        r |= mq.decode(ctx, tbl, 17);
                        const uint32_t si = T.sc[sc_index(wl, sl, wc, sc, wr, sr, r)];
                        const uint32_t neg = (uint32_t)mq.decode(ctx, tbl, si & 15) ^ (si >> 4);
                        wc |= 2u << r;
                        sc |= neg << (r + 1);
                        S.mag[(4 * s + r) * 64 + c] = pbit;
                        k = r + 1;
                    }
                }
                if (!run_done) {
                    for (; k < rows; k++) {
                        if (((wc >> (k + 1)) | (vis >> k)) & 1u) continue;
                        if (mq.decode(ctx, tbl, zc[zc_pattern(wl, wc, wr, k)])) {
                            const uint32_t si = T.sc[sc_index(wl, sl, wc, sc, wr, sr, k)];
                            const uint32_t neg = (uint32_t)mq.decode(ctx, tbl, si & 15) ^ (si >> 4);
                            wc |= 2u << k;
                            sc |= neg << (k + 1);
                            S.mag[(4 * s + k) * 64 + c] = pbit;
                        }
                    }
                }
                if (wc != wc0) {
                    S.sig[c + 1] |= (unsigned long long)((wc >> 1) & 0xFu) << (4 * s);
                    S.sgn[c + 1] |= (unsigned long long)((sc >> 1) & 0xFu) << (4 * s);
                }
                wl = wc;
                sl = sc;
                wc = wr;
                sc = sr;
            }
        }
        type = 0;
        *last_plane = p;
        if (++pass >= passes) break;
        for (int c = 0; c < kCols; c++) S.vis[c] = 0ull;
    }
    return type;
}

__global__ void __launch_bounds__(32 * kWarps)
t1_decode_kernel(const tc_cblk_desc *__restrict__ desc, const uint32_t *__restrict__ order, int n,
                 const uint8_t *__restrict__ pool, uint64_t pool_len, char *__restrict__ out,
                 int out_mode, float recon_r, uint32_t *words)
{
    extern __shared__ __align__(16) unsigned char smem[];
    Tables &T = *reinterpret_cast<Tables *>(smem);
    WarpState *states = reinterpret_cast<WarpState *>(smem + ((sizeof(Tables) + 15) & ~size_t(15)));
    build_tables(T);
    __syncthreads();

    const int lane = threadIdx.x & 31;
    WarpState &S = states[threadIdx.x >> 5];

    for (;;) {
        int idx = 0;
        if (lane == 0) idx = (int)atomicAdd(&words[1], 1u);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= n) break;
        const uint32_t bi = order ? order[idx] : (uint32_t)idx;
        if (bi >= (uint32_t)n) {
            if (lane == 0) atomicOr(&words[0], TC_DERR_DESC);
            continue;
        }
        const tc_cblk_desc d = desc[bi];
        const int w = d.w, h = d.h;
        const bool geom_ok = w >= 1 && w <= 64 && h >= 1 && h <= 64;
        const int numbps = (int)d.mb - (int)d.zero_bitplanes;
        bool ok = geom_ok && d.mb >= 1 && d.mb <= 31 && d.orient <= 3 && numbps >= 0 &&
                  (numbps == 0 || d.passes <= 3 * numbps - 2);
        const bool pool_ok = d.seg_off <= pool_len && (uint64_t)d.seg_len <= pool_len - d.seg_off;
        if (!geom_ok) {
            if (lane == 0) atomicOr(&words[0], TC_DERR_DESC);
            continue;
        }
        if (!ok || !pool_ok) {
            if (lane == 0) atomicOr(&words[0], ok ? TC_DERR_POOL : TC_DERR_DESC);
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
        if (coded && lane == 0)
            type = decode_block(S, T, pool + d.seg_off, (int)d.seg_len, w, h, d.orient, numbps,
                                d.passes, &last_plane);
        type = __shfl_sync(0xffffffffu, type, 0);
        last_plane = __shfl_sync(0xffffffffu, last_plane, 0);
        __syncwarp();

        // epilogue: reconstruction + inverse quantisation, coalesced rows
        const bool irrev = (d.flags & TC_CBLK_IRREVERSIBLE) != 0;
        for (int y = 0; y < h; y++) {
            char *row = out + 4 * (d.out_off + (uint64_t)y * d.out_pitch);
            for (int x = lane; x < w; x += 32) {
                const bool sg = coded && ((S.sig[x + 1] >> y) & 1ull);
                uint32_t mg = 0, neg = 0, u = 0;
                if (sg) {
                    mg = S.mag[y * 64 + x];
                    neg = (uint32_t)(S.sgn[x + 1] >> y) & 1u;
                    u = (uint32_t)last_plane;
                    if (type == 1 && !((S.vis[x + 1] >> y) & 1ull)) u++;
                }
                if (out_mode == TC_T1_OUT_RAW) {
                    reinterpret_cast<uint32_t *>(row)[x] = sg ? ((mg << (31 - d.mb)) | (neg << 31)) : 0u;
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

cudaError_t launch_t1_decode(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order, int n,
                             const uint8_t *d_pool, uint64_t pool_len, void *d_out, int out_mode,
                             float recon_r)
{
    if (n <= 0) return cudaSuccess;
    const size_t smem = ((sizeof(Tables) + 15) & ~size_t(15)) + kWarps * sizeof(WarpState);
    static bool attr_done[64] = {};
    if (ctx->device >= 0 && ctx->device < 64 && !attr_done[ctx->device]) {
        cudaError_t e = cudaFuncSetAttribute(t1_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_done[ctx->device] = true;
    }
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, t1_decode_kernel, 32 * kWarps, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const int want = (n + kWarps - 1) / kWarps;
    const int grid = std::min(want, per_sm * num_sms(ctx->device));
    e = cudaMemsetAsync(ctx->d_words + 1, 0, sizeof(uint32_t), ctx->stream);
    if (e != cudaSuccess) return e;
    t1_decode_kernel<<<grid, 32 * kWarps, smem, ctx->stream>>>(d_desc, d_order, n, d_pool, pool_len,
                                                               static_cast<char *>(d_out), out_mode,
                                                               recon_r, ctx->d_words);
    ctx->launches++;
    return cudaGetLastError();
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
