// capi.cu -- the extern "C" boundary of libtc_j2k (see include/tc_j2k.h).
//
// Orchestrates the decode the reference's Decoder::decode performs
// (Decoder.cpp:94-217) on one CUDA stream per context:
//   parse (host) -> H2D segment pool + descriptors -> Tier-1 with fused
//   dequantisation (one persistent launch over every code-block of every
//   image) -> reverse DWT levels (ping-pong scratch, no LL copies) -> last
//   level fused with inverse colour / DC shift / clamp -> D2H.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "j2k_host.h"
#include "tc_internal.cuh"

namespace tc {

cudaError_t DevBuf::ensure(size_t bytes)
{
    if (bytes <= size && ptr) return cudaSuccess;
    // Grow by at least half again: a serving loop whose batches vary in size
    // reallocates (and so synchronises the device in cudaFree) only rarely.
    const size_t want = std::max<size_t>(std::max<size_t>(bytes, 256), size + size / 2);
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    size = 0;
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e == cudaSuccess) size = want;
    else ptr = nullptr;
    return e;
}

cudaError_t ctx_mem_pool(tc_ctx *ctx, cudaMemPool_t *out)
{
    if (!ctx->pool) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ctx->device;
        cudaMemPool_t p = nullptr;
        cudaError_t e = cudaMemPoolCreate(&p, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = ~uint64_t(0);
        e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(p);
            return e;
        }
        ctx->pool = p;
    }
    *out = ctx->pool;
    return cudaSuccess;
}

cudaError_t DevBuf::ensure_on(size_t bytes, cudaStream_t s, cudaMemPool_t pool)
{
    if (bytes <= size && ptr) return cudaSuccess;
    const size_t want = std::max<size_t>(std::max<size_t>(bytes, 256), size + size / 2);
    if (ptr) {
        if (ordered) cudaFreeAsync(ptr, stream);
        else cudaFree(ptr);
    }
    ptr = nullptr;
    size = 0;
    cudaError_t e = cudaMallocFromPoolAsync(&ptr, want, pool, s);
    if (e == cudaSuccess) {
        size = want;
        stream = s;
        ordered = true;
    } else {
        ptr = nullptr;
    }
    return e;
}

void DevBuf::release()
{
    if (ptr) {
        if (ordered) {
            cudaFreeAsync(ptr, stream);
            cudaStreamSynchronize(stream);
        } else {
            cudaFree(ptr);
        }
    }
    ptr = nullptr;
    size = 0;
    ordered = false;
}

cudaError_t ensure_side_streams(tc_ctx *ctx)
{
    if (ctx->side[0]) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaStreamCreateWithFlags(&ctx->side[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->capture, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming);
    return e;
}

int fail(tc_ctx *ctx, int status, const std::string &msg)
{
    if (ctx) ctx->err = msg;
    return status;
}

int cuda_status(tc_ctx *ctx, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return TC_OK;
    if (e == cudaErrorMemoryAllocation) return fail(ctx, TC_E_OOM, std::string(what) + ": out of device memory");
    return fail(ctx, TC_E_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}

static int check_ctx(tc_ctx *ctx)
{
    if (!ctx) return TC_E_ARG;
    cudaError_t e = cudaSetDevice(ctx->device);
    return cuda_status(ctx, e, "cudaSetDevice");
}

static int sample_bytes(int bits) { return bits <= 8 ? 1 : 2; }
// The `bits` argument of the output stages: the depth, TC_SIGNED for signed samples.
static int out_bits(const tc_image_info &inf) { return inf.bits | (inf.is_signed ? TC_SIGNED : 0); }
// Whether the image has subsampled components, and component c's plane size.
static bool subsampled(const tc_image_info &inf)
{
    for (int c = 0; c < inf.ncomp && c < 4; c++)
        if (inf.comp_dx[c] > 1 || inf.comp_dy[c] > 1) return true;
    return false;
}
static void comp_size(const tc_image_info &inf, int c, int *w, int *h)
{
    const int dx = inf.comp_dx[c] ? inf.comp_dx[c] : 1, dy = inf.comp_dy[c] ? inf.comp_dy[c] : 1;
    *w = (inf.width + dx - 1) / dx;
    *h = (inf.height + dy - 1) / dy;
}
// Samples of all components (planar, each at its own size).
static size_t image_samples(const tc_image_info &inf)
{
    size_t n = 0;
    for (int c = 0; c < inf.ncomp; c++) {
        int w, h;
        comp_size(inf, c, &w, &h);
        n += (size_t)w * h;
    }
    return n;
}

// Reverse DWT of ncomp components from Mallat planes coef[c] (pitch cp)
// through levels >= 2 into ping-pong scratch, and the last level either into
// T planes (out_color < 0) or fused with colour into out_type samples.
static int run_reverse(tc_ctx *ctx, int wavelet, int rounding, const void *const *coef, int cp, int w, int h,
                       int levels, int ncomp, char *scratch, void *const *out, int out_pitch, int color,
                       int out_type, int bits)
{
    std::vector<int> ws, hs;
    level_sizes(w, h, levels, ws, hs);
    const size_t esz = 4;
    const size_t sw = levels >= 1 ? ws[1] : 0, sh = levels >= 1 ? hs[1] : 0;
    const size_t slab = sw * sh * esz;  // one intermediate plane
    const void *src[4];
    int src_pitch = cp;
    for (int c = 0; c < ncomp; c++) src[c] = coef[c];
    for (int l = levels; l >= 1; l--) {
        LevelIO io{};
        io.w = ws[l - 1];
        io.h = hs[l - 1];
        io.ncomp = ncomp;
        io.ll_pitch = src_pitch;
        io.coef_pitch = cp;
        for (int c = 0; c < ncomp; c++) {
            io.ll[c] = src[c];
            io.coef[c] = coef[c];
        }
        if (l == 1) {
            io.out_pitch = out_pitch;
            for (int c = 0; c < ncomp; c++) io.out[c] = out[c];
            cudaError_t e = color >= 0 ? launch_idwt_last_color(ctx, io, wavelet, color, out_type, bits, true)
                                       : launch_idwt_level(ctx, io, wavelet, rounding);
            if (e != cudaSuccess) return cuda_status(ctx, e, "reverse DWT (last level)");
        } else {
            const int buf = (levels - l) & 1;
            io.out_pitch = (int)sw;
            for (int c = 0; c < ncomp; c++) io.out[c] = scratch + ((size_t)c * 2 + buf) * slab;
            cudaError_t e = launch_idwt_level(ctx, io, wavelet, rounding);
            if (e != cudaSuccess) return cuda_status(ctx, e, "reverse DWT");
            for (int c = 0; c < ncomp; c++) src[c] = io.out[c];
            src_pitch = (int)sw;
        }
    }
    return TC_OK;
}

void t1_class_order(const tc_cblk_desc *h_desc, int n, uint32_t *h_order, int counts[6])
{
    std::vector<uint32_t> all(n);
    tc_t1_sort_order(h_desc, n, all.data());
    std::vector<uint32_t> cls[6];
    for (uint32_t i : all) {
        const tc_cblk_desc &d = h_desc[i];
        const int nb = d.passes ? (int)d.mb - (int)d.zero_bitplanes : 0;
        const int k = (nb <= 8 ? 0 : (nb <= 16 ? 1 : 2)) + ((d.style & kStyleDecodeBits) ? 3 : 0);
        cls[k].push_back(i);
    }
    int o = 0;
    for (int k = 0; k < 6; k++) {
        counts[k] = (int)cls[k].size();
        for (uint32_t i : cls[k]) h_order[o++] = i;
    }
}

static size_t reverse_scratch_bytes(int w, int h, int levels, int ncomp)
{
    if (levels < 2) return 0;
    return (size_t)ncomp * 2 * (size_t)((w + 1) / 2) * (size_t)((h + 1) / 2) * 4;
}

}  // namespace tc

using namespace tc;

// ============================ plan ===========================================

struct tc_plan {
    tc_ctx *ctx = nullptr;
    struct Img {
        tc_image_info info{};
        uint64_t coef_off = 0;     // byte offset in the coefficient arena
        size_t out_bytes = 0;
        std::vector<tc_tile_info> tiles;  // tile-major coefficients from coef_off
        std::vector<size_t> tile_scratch; // each tile's scratch, from the image's
        size_t comp_scratch[4] = {0, 0, 0, 0};  // subsampled images: each component's scratch
    };
    std::vector<Img> imgs;
    DevBuf pool, desc, order, coef, scratch;
    int ncblk = 0;
    uint64_t pool_len = 0;
    size_t scratch_per_img = 0;
    // batched reverse DWT (plans of several images): each image's own
    // scratch region, and the job table of the level launches for the
    // output buffers it was built for
    std::vector<size_t> scratch_off;
    struct DwtLaunch {
        int first, njobs, ntiles, wavelet, color, ncomp, otype, bits;
    };
    std::vector<DwtLaunch> dwt_launches;
    std::vector<void *> jobs_outs;
    PinBuf h_jobs;
    DevBuf jobs;
    cudaEvent_t jobs_uploaded = nullptr;
    float recon_r = 0.5f;
    // a single image's segment pool already uploaded from pinned memory
    // (tc_decode_j2k): its host address and length
    const void *preloaded = nullptr;
    uint64_t preloaded_len = 0;
    int class_counts[6] = {0, 0, 0, 0, 0, 0};  // Tier-1 blocks of <= 8, <= 16, <= 31 coded bit-planes; styled ones alike
    bool profiling = false;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    PinBuf h_pool, h_desc, h_order;  // pinned host staging, alive until the next build
    // Graph replay of execute (tc_plan_set_graph), one graph per shape
    // bucket.  A graph's kernels read everything that varies with the
    // images (descriptors, order, segment pool, DWT job table with the
    // output pointers) from plan buffers, so it is keyed by its launch
    // parameters: buffer addresses, Tier-1 class sizes and the DWT launch
    // list.  Another batch of the same launch topology (same classes and
    // DWT launch kinds) updates a cached graph's parameters in place
    // (cudaGraphExecUpdate) instead of instantiating a new one.
    struct Graph {
        std::vector<uint64_t> key, topo;
        cudaGraphExec_t exec = nullptr;
        uint64_t launches = 0, last_use = 0;
    };
    bool use_graph = false;
    std::vector<Graph> graphs;      // at most kMaxGraphs, least recently used dropped
    uint64_t graph_tick = 0;
    uint64_t graph_captures = 0, graph_updates = 0, graph_replays = 0;
};

static constexpr size_t kMaxGraphs = 8;

// Plans of several images or of tiled images run the batched reverse DWT.
static bool plan_batched(const tc_plan *P)
{
    return P->imgs.size() > 1 ||
           (P->imgs.size() == 1 && (P->imgs[0].tiles.size() > 1 || subsampled(P->imgs[0].info)));
}

static void plan_drop_graphs(tc_plan *P)
{
    for (tc_plan::Graph &g : P->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    P->graphs.clear();
}

// Lays out and uploads a batch from parsed images: parsed[i] with its
// segment pool pools[i] of pool_lens[i] bytes (the codestream itself for
// single-layer streams).
static int plan_build_parsed(tc_ctx *ctx, const Parsed *const *parsed, const uint8_t *const *pools,
                             const uint64_t *pool_lens, int n, tc_plan *P)
{
    P->ctx = ctx;
    P->imgs.clear();
    P->ncblk = 0;
    uint64_t pool_total = 0, coef_total = 0;
    size_t scratch_max = 0, scratch_sum = 0;
    P->scratch_off.clear();
    P->jobs_outs.clear();
    for (int i = 0; i < n; i++) {
        const tc_image_info &inf = parsed[i]->info;
        P->scratch_off.push_back(scratch_sum);
        tc_plan::Img im;
        im.info = inf;
        im.coef_off = coef_total;
        coef_total += (uint64_t)image_samples(inf) * 4;
        coef_total = (coef_total + 255) & ~uint64_t(255);
        im.out_bytes = image_samples(inf) * sample_bytes(inf.bits);
        im.tiles = parsed[i]->tiles;
        size_t img_scratch = 0;
        if (subsampled(inf)) {
            for (int c = 0; c < inf.ncomp; c++) {
                int cw, ch;
                comp_size(inf, c, &cw, &ch);
                im.comp_scratch[c] = img_scratch;
                img_scratch += (reverse_scratch_bytes(cw, ch, inf.levels, 1) + 255) & ~size_t(255);
            }
        } else {
            for (const tc_tile_info &t : im.tiles) {
                im.tile_scratch.push_back(img_scratch);
                img_scratch += (reverse_scratch_bytes(t.w, t.h, inf.levels, inf.ncomp) + 255) & ~size_t(255);
            }
        }
        scratch_max = std::max(scratch_max, img_scratch);
        scratch_sum += img_scratch;
        P->imgs.push_back(im);
        pool_total += (pool_lens[i] + 15) & ~uint64_t(15);
        P->ncblk += (int)parsed[i]->desc.size();
    }
    // Pinned host staging (the plan keeps it until its next build, so the
    // uploads below are asynchronous): pool and rebased descriptors.
    cudaError_t e;
    // the previous execute may still read the staging through its uploads
    if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) return cuda_status(ctx, e, "plan staging");
    const size_t pool_bytes = pool_total ? pool_total : 16;
    if ((e = P->h_pool.ensure(pool_bytes)) != cudaSuccess ||
        (e = P->h_desc.ensure(sizeof(tc_cblk_desc) * std::max(1, P->ncblk))) != cudaSuccess ||
        (e = P->h_order.ensure(sizeof(uint32_t) * std::max(1, P->ncblk))) != cudaSuccess)
        return cuda_status(ctx, e, "plan staging");
    uint8_t *hpool = static_cast<uint8_t *>(P->h_pool.ptr);
    tc_cblk_desc *hdesc = static_cast<tc_cblk_desc *>(P->h_desc.ptr);
    uint32_t *horder = static_cast<uint32_t *>(P->h_order.ptr);
    const bool preloaded = n == 1 && P->preloaded && pools[0] == P->preloaded && pool_lens[0] == P->preloaded_len;
    P->preloaded = nullptr;
    uint64_t po = 0;
    size_t nd = 0;
    for (int i = 0; i < n; i++) {
        const uint64_t pl = pool_lens[i];
        if (pl && !preloaded) std::memcpy(hpool + po, pools[i], pl);
        const uint64_t elem_base = P->imgs[i].coef_off / 4;
        for (tc_cblk_desc d : parsed[i]->desc) {
            d.seg_off += po;
            d.out_off += elem_base;
            hdesc[nd++] = d;
        }
        po += (pl + 15) & ~uint64_t(15);
    }
    t1_class_order(hdesc, P->ncblk, horder, P->class_counts);
    P->pool_len = pool_total;
    P->scratch_per_img = scratch_max;
    cudaStream_t st = ctx->stream;
    cudaMemPool_t mp = nullptr;
    if ((e = ctx_mem_pool(ctx, &mp)) != cudaSuccess ||
        (e = P->pool.ensure_on(pool_bytes, st, mp)) != cudaSuccess ||
        (e = P->desc.ensure_on(sizeof(tc_cblk_desc) * std::max(1, P->ncblk), st, mp)) != cudaSuccess ||
        (e = P->order.ensure_on(sizeof(uint32_t) * std::max(1, P->ncblk), st, mp)) != cudaSuccess ||
        (e = P->coef.ensure_on(std::max<uint64_t>(coef_total, 256), st, mp)) != cudaSuccess ||
        (e = P->scratch.ensure_on(std::max<size_t>(plan_batched(P) ? scratch_sum : scratch_max, 256), st, mp)) !=
            cudaSuccess)
        return cuda_status(ctx, e, "plan allocation");
    if ((!preloaded &&
         (e = cudaMemcpyAsync(P->pool.ptr, hpool, pool_bytes, cudaMemcpyHostToDevice, ctx->stream))) ||
        (e = cudaMemcpyAsync(P->desc.ptr, hdesc, sizeof(tc_cblk_desc) * P->ncblk, cudaMemcpyHostToDevice,
                             ctx->stream)) ||
        (e = cudaMemcpyAsync(P->order.ptr, horder, sizeof(uint32_t) * P->ncblk, cudaMemcpyHostToDevice,
                             ctx->stream)))
        return cuda_status(ctx, e, "plan upload");
    return TC_OK;
}

static int plan_build(tc_ctx *ctx, const uint8_t *const *cs, const size_t *lens, int n, tc_plan *P)
{
    std::vector<Parsed> parsed(n);
    std::vector<const Parsed *> pp(n);
    std::vector<const uint8_t *> pools(n);
    std::vector<uint64_t> plens(n);
    std::string err;
    for (int i = 0; i < n; i++) {
        if (!cs[i] || !lens[i]) return fail(ctx, TC_E_ARG, "empty codestream");
        const int rc = parse_codestream(cs[i], lens[i], parsed[i], err);
        if (rc) return fail(ctx, rc, "image " + std::to_string(i) + ": " + err);
        pp[i] = &parsed[i];
        pools[i] = parsed[i].pool_is_cs ? cs[i] : parsed[i].own_pool.data();
        plens[i] = parsed[i].pool_is_cs ? lens[i] : parsed[i].own_pool.size();
    }
    return plan_build_parsed(ctx, pp.data(), pools.data(), plens.data(), n, P);
}

// Reverse DWT of every tile of every image of a plan with one launch per
// level step and kind instead of per tile and level: at step t a tile of an
// image of L levels runs its level L - t, so tiles and images of different
// sizes and level counts share the launches.  Intermediate levels are
// grouped by wavelet (each job one component plane of one tile); last
// levels, fused with colour and written into the image at the tile's
// position, by wavelet, colour transform, component count, sample type and
// bit depth.  The job table is built on the host and uploaded once per set
// of output buffers (a replayed graph needs no copy).
static int run_reverse_batched(tc_plan *P, void *const *d_out, bool launch = true)
{
    tc_ctx *ctx = P->ctx;
    const size_t nimg = P->imgs.size();
    std::vector<void *> outs(d_out, d_out + nimg);
    cudaError_t e;
    auto color_of = [](const tc_image_info &inf) {
        return inf.mct && inf.ncomp >= 3 ? (inf.reversible ? TC_COLOR_RCT : TC_COLOR_ICT) : TC_COLOR_DC;
    };
    // one reverse transform: a tile of an image (an untiled image is one
    // tile), or one component of an image whose components are subsampled
    struct Unit {
        const tc_image_info *inf;
        int w, h, ncomp, color;
        void *coef[4];   // the unit's component planes, pitch w
        void *out[4];    // the unit's first sample in each output plane
        int out_pitch;
        char *scratch;
    };
    std::vector<Unit> units;
    for (size_t i = 0; i < nimg; i++) {
        const tc_plan::Img &im = P->imgs[i];
        const tc_image_info &inf = im.info;
        char *coef = static_cast<char *>(P->coef.ptr) + im.coef_off;
        char *out = static_cast<char *>(d_out[i]);
        char *scratch = static_cast<char *>(P->scratch.ptr) + P->scratch_off[i];
        const size_t plane = (size_t)inf.width * inf.height;
        const int ob = sample_bytes(inf.bits);
        if (subsampled(inf)) {
            size_t off = 0;  // the parser's and the output's planar order
            for (int c = 0; c < inf.ncomp; c++) {
                Unit u{};
                u.inf = &inf;
                comp_size(inf, c, &u.w, &u.h);
                u.ncomp = 1;
                u.color = TC_COLOR_DC;
                u.coef[0] = coef + off * 4;
                u.out[0] = out + off * ob;
                u.out_pitch = u.w;
                u.scratch = scratch + im.comp_scratch[c];
                units.push_back(u);
                off += (size_t)u.w * u.h;
            }
            continue;
        }
        for (size_t k = 0; k < im.tiles.size(); k++) {
            const tc_tile_info &t = im.tiles[k];
            Unit u{};
            u.inf = &inf;
            u.w = t.w;
            u.h = t.h;
            u.ncomp = inf.ncomp;
            u.color = color_of(inf);
            for (int c = 0; c < inf.ncomp; c++) {
                u.coef[c] = coef + (t.coef_off + (size_t)c * t.w * t.h) * 4;
                u.out[c] = out + ((size_t)c * plane + (size_t)t.y0 * inf.width + t.x0) * ob;
            }
            u.out_pitch = inf.width;
            u.scratch = scratch + im.tile_scratch[k];
            units.push_back(u);
        }
    }
    const size_t nu = units.size();
    // images without a transform: colour only
    for (const Unit &u : units) {
        const tc_image_info &inf = *u.inf;
        if (inf.levels || !launch) continue;
        const int ob = sample_bytes(inf.bits);
        e = launch_color_inverse(ctx, u.color, u.ncomp, u.coef, inf.reversible ? TC_INT32 : TC_FLOAT32, u.w, u.out,
                                 ob == 1 ? TC_U8 : TC_U16, u.out_pitch, u.w, u.h, out_bits(inf));
        if (e != cudaSuccess) return cuda_status(ctx, e, "colour");
    }
    if (outs != P->jobs_outs) {
        std::vector<RevJob> jobs;
        std::vector<tc_plan::DwtLaunch> launches;
        struct Walk {
            std::vector<int> ws, hs;
            const void *src[4];
            int src_pitch;
            size_t slab;
        };
        std::vector<Walk> wk(nu);
        int maxl = 0;
        for (size_t i = 0; i < nu; i++) {
            const Unit &u = units[i];
            Walk &W = wk[i];
            level_sizes(u.w, u.h, u.inf->levels, W.ws, W.hs);
            for (int c = 0; c < u.ncomp; c++) W.src[c] = u.coef[c];
            W.src_pitch = u.w;
            W.slab = u.inf->levels >= 1 ? (size_t)W.ws[1] * W.hs[1] * 4 : 0;
            maxl = std::max(maxl, u.inf->levels);
        }
        for (int t = 0; t < maxl; t++) {
            // intermediate levels, by wavelet
            for (int wv = 0; wv < 2; wv++) {
                const int first = (int)jobs.size();
                int tiles = 0, tx, ty;
                rev_tile_shape(wv, &tx, &ty);
                for (size_t i = 0; i < nu; i++) {
                    const Unit &u = units[i];
                    const tc_image_info &inf = *u.inf;
                    const int l = inf.levels - t;
                    if (l < 2 || (inf.reversible ? 0 : 1) != wv) continue;
                    Walk &W = wk[i];
                    const int buf = (inf.levels - l) & 1;
                    for (int c = 0; c < u.ncomp; c++) {
                        RevJob J{};
                        J.io.w = W.ws[l - 1];
                        J.io.h = W.hs[l - 1];
                        J.io.ncomp = 1;
                        J.io.ll[0] = W.src[c];
                        J.io.ll_pitch = W.src_pitch;
                        J.io.coef[0] = u.coef[c];
                        J.io.coef_pitch = u.w;
                        J.io.out[0] = u.scratch + ((size_t)c * 2 + buf) * W.slab;
                        J.io.out_pitch = W.ws[1];
                        J.tiles_x = (J.io.w + tx - 1) / tx;
                        J.tile0 = tiles;
                        tiles += J.tiles_x * ((J.io.h + ty - 1) / ty);
                        jobs.push_back(J);
                    }
                    for (int c = 0; c < u.ncomp; c++) W.src[c] = u.scratch + ((size_t)c * 2 + buf) * W.slab;
                    W.src_pitch = W.ws[1];
                }
                if ((int)jobs.size() > first)
                    launches.push_back({first, (int)jobs.size() - first, tiles, wv, -1, 1, 0, 0});
            }
            // last levels with colour, by kernel instance
            std::vector<char> taken(nu, 0);
            for (size_t i0 = 0; i0 < nu; i0++) {
                const Unit &ua = units[i0];
                const tc_image_info &a = *ua.inf;
                if (taken[i0] || a.levels - t != 1) continue;
                const int first = (int)jobs.size();
                int tiles = 0, tx, ty;
                const int wv = a.reversible ? 0 : 1;
                rev_tile_shape(wv, &tx, &ty);
                for (size_t i = i0; i < nu; i++) {
                    const Unit &u = units[i];
                    const tc_image_info &inf = *u.inf;
                    if (taken[i] || inf.levels - t != 1 || inf.reversible != a.reversible || u.color != ua.color ||
                        u.ncomp != ua.ncomp || sample_bytes(inf.bits) != sample_bytes(a.bits) ||
                        out_bits(inf) != out_bits(a))
                        continue;
                    taken[i] = 1;
                    Walk &W = wk[i];
                    RevJob J{};
                    J.io.w = W.ws[0];
                    J.io.h = W.hs[0];
                    J.io.ncomp = u.ncomp;
                    J.io.ll_pitch = W.src_pitch;
                    J.io.coef_pitch = u.w;
                    J.io.out_pitch = u.out_pitch;
                    for (int c = 0; c < u.ncomp; c++) {
                        J.io.ll[c] = W.src[c];
                        J.io.coef[c] = u.coef[c];
                        J.io.out[c] = u.out[c];
                    }
                    J.tiles_x = (J.io.w + tx - 1) / tx;
                    J.tile0 = tiles;
                    tiles += J.tiles_x * ((J.io.h + ty - 1) / ty);
                    jobs.push_back(J);
                }
                launches.push_back({first, (int)jobs.size() - first, tiles, wv, ua.color, ua.ncomp,
                                    sample_bytes(a.bits) == 1 ? TC_U8 : TC_U16, out_bits(a)});
            }
        }
        // the previous table's upload must be done before its staging is rewritten
        if (P->jobs_uploaded && (e = cudaEventSynchronize(P->jobs_uploaded)) != cudaSuccess)
            return cuda_status(ctx, e, "DWT job table");
        const size_t bytes = std::max<size_t>(jobs.size(), 1) * sizeof(RevJob);
        cudaMemPool_t mp = nullptr;
        if ((e = P->h_jobs.ensure(bytes)) != cudaSuccess || (e = ctx_mem_pool(ctx, &mp)) != cudaSuccess ||
            (e = P->jobs.ensure_on(bytes, ctx->stream, mp)) != cudaSuccess)
            return cuda_status(ctx, e, "DWT job table");
        if (!jobs.empty()) std::memcpy(P->h_jobs.ptr, jobs.data(), jobs.size() * sizeof(RevJob));
        if (!P->jobs_uploaded && (e = cudaEventCreateWithFlags(&P->jobs_uploaded, cudaEventDisableTiming)) !=
                                     cudaSuccess)
            return cuda_status(ctx, e, "DWT job table");
        if ((e = cudaMemcpyAsync(P->jobs.ptr, P->h_jobs.ptr, jobs.size() * sizeof(RevJob), cudaMemcpyHostToDevice,
                                 ctx->stream)) != cudaSuccess ||
            (e = cudaEventRecord(P->jobs_uploaded, ctx->stream)) != cudaSuccess)
            return cuda_status(ctx, e, "DWT job table");
        P->dwt_launches = launches;
        P->jobs_outs = outs;
    }
    if (!launch) return TC_OK;
    const RevJob *dj = static_cast<const RevJob *>(P->jobs.ptr);
    for (const tc_plan::DwtLaunch &L : P->dwt_launches) {
        e = launch_idwt_batch(ctx, dj + L.first, L.njobs, L.ntiles, L.wavelet, TC_ROUND_FLOOR, L.color, L.ncomp,
                              L.otype, L.bits);
        if (e != cudaSuccess) return cuda_status(ctx, e, "reverse DWT (batched)");
    }
    return TC_OK;
}

// One execute's launches.  In graph mode every plan takes the batched
// reverse DWT (its output pointers then sit in the job table, not in kernel
// parameters) and Tier-1 bounds codewords by the pool buffer's capacity
// rather than this batch's exact pool length, so that the launch parameters
// depend on the batch's shape only.
static int plan_run(tc_plan *P, void *const *d_out, bool graph_mode = false)
{
    tc_ctx *ctx = P->ctx;
    if (P->profiling) cudaEventRecord(P->ev[0], ctx->stream);
    cudaError_t e = launch_t1_classes(ctx, static_cast<tc_cblk_desc *>(P->desc.ptr),
                                      static_cast<uint32_t *>(P->order.ptr), P->ncblk, P->class_counts[0],
                                      P->class_counts[1], P->class_counts[2],
                                      static_cast<uint8_t *>(P->pool.ptr), graph_mode ? P->pool.size : P->pool_len,
                                      P->coef.ptr, P->coef.size / 4, TC_T1_OUT_DEQUANT, P->recon_r,
                                      P->class_counts + 3);
    if (e != cudaSuccess) return cuda_status(ctx, e, "Tier-1 launch");
    if (P->profiling) cudaEventRecord(P->ev[1], ctx->stream);
    if (graph_mode || plan_batched(P)) {
        const int rc = run_reverse_batched(P, d_out);
        if (rc) return rc;
        if (P->profiling) cudaEventRecord(P->ev[2], ctx->stream);
        return TC_OK;
    }
    for (size_t i = 0; i < P->imgs.size(); i++) {
        const tc_image_info &inf = P->imgs[i].info;
        char *coef = static_cast<char *>(P->coef.ptr) + P->imgs[i].coef_off;
        const size_t plane = (size_t)inf.width * inf.height;
        const int ob = sample_bytes(inf.bits);
        void *cptr[4], *optr[4];
        for (int c = 0; c < inf.ncomp; c++) {
            cptr[c] = coef + (size_t)c * plane * 4;
            optr[c] = static_cast<char *>(d_out[i]) + (size_t)c * plane * ob;
        }
        const int color = inf.mct && inf.ncomp >= 3 ? (inf.reversible ? TC_COLOR_RCT : TC_COLOR_ICT) : TC_COLOR_DC;
        const int wavelet = inf.reversible ? 0 : 1;
        const int otype = ob == 1 ? TC_U8 : TC_U16;
        int rc;
        if (inf.levels == 0) {
            e = launch_color_inverse(ctx, color, inf.ncomp, cptr, inf.reversible ? TC_INT32 : TC_FLOAT32,
                                     inf.width, optr, otype, inf.width, inf.width, inf.height, out_bits(inf));
            rc = cuda_status(ctx, e, "colour");
        } else {
            rc = run_reverse(ctx, wavelet, TC_ROUND_FLOOR, cptr, inf.width, inf.width, inf.height, inf.levels,
                             inf.ncomp, static_cast<char *>(P->scratch.ptr), optr, inf.width, color, otype,
                             out_bits(inf));
        }
        if (rc) return rc;
    }
    if (P->profiling) cudaEventRecord(P->ev[2], ctx->stream);
    return TC_OK;
}

// ============================ C ABI ==========================================

extern "C" {

int tc_version(void) { return 10000; }

const char *tc_status_string(int s)
{
    switch (s) {
    case TC_OK: return "ok";
    case TC_E_ARG: return "invalid argument";
    case TC_E_OOM: return "out of memory";
    case TC_E_CODESTREAM: return "malformed codestream";
    case TC_E_DEVICE: return "CUDA error";
    case TC_E_TIMEOUT: return "device wait timed out";
    case TC_E_UNSUPPORTED: return "unsupported codestream feature";
    case TC_E_NOFILE: return "file not found";
    default: return "unknown status";
    }
}

int tc_ctx_create(int device, void *cuda_stream, tc_ctx **out)
{
    if (!out) return TC_E_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return TC_E_DEVICE;
    tc_ctx *ctx = new (std::nothrow) tc_ctx;
    if (!ctx) return TC_E_OOM;
    ctx->device = device;
    ctx->stream = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_words, 8 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(ctx->d_words, 0, 8 * sizeof(uint32_t));
    if (e != cudaSuccess) {
        delete ctx;
        return e == cudaErrorMemoryAllocation ? TC_E_OOM : TC_E_DEVICE;
    }
    *out = ctx;
    return TC_OK;
}

int tc_ctx_destroy(tc_ctx *ctx)
{
    if (!ctx) return TC_E_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->scratch.release();
    ctx->tmp_pool.release();
    ctx->tmp_desc.release();
    ctx->tmp_order.release();
    ctx->tmp_coef.release();
    ctx->tmp_out.release();
    ctx->stage_pool.release();
    ctx->stage_desc.release();
    ctx->stage_order.release();
    ctx->tmp_jobs.release();
    for (auto &b : ctx->enc) b.release();
    ctx->enc_host.release();
    ctx->stage_jobs.release();
    if (ctx->jobs_uploaded) cudaEventDestroy(ctx->jobs_uploaded);
    if (ctx->d_words) cudaFree(ctx->d_words);
    for (int i = 0; i < 2; i++) {
        if (ctx->side[i]) cudaStreamDestroy(ctx->side[i]);
        if (ctx->ev_join[i]) cudaEventDestroy(ctx->ev_join[i]);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->capture) cudaStreamDestroy(ctx->capture);
    // buffers still drawn from the pool (plans not destroyed yet) keep it
    // alive until they are freed
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
    return TC_OK;
}

int tc_ctx_synchronize(tc_ctx *ctx)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_status(ctx, e, "synchronize");
    uint32_t w = 0;
    e = cudaMemcpy(&w, ctx->d_words, sizeof w, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(ctx, e, "read device error word");
    if (w) {
        cudaMemset(ctx->d_words, 0, sizeof w);
        return fail(ctx, (w & TC_DERR_TIMEOUT) ? TC_E_TIMEOUT : TC_E_CODESTREAM,
                    (w & TC_DERR_TIMEOUT) ? "a bounded device wait for a TMA copy gave up"
                    : (w & TC_DERR_OUT)   ? "a code-block's place runs past the output (the block was skipped)"
                    : (w & TC_DERR_POOL)  ? "a code-block codeword runs past the segment pool"
                    : (w & TC_DERR_STYLE) ? "a code-block style this launch does not decode, or a bad segment table"
                                          : "a code-block descriptor is out of range");
    }
    return TC_OK;
}

const char *tc_ctx_last_error(const tc_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

uint64_t tc_ctx_launch_count(const tc_ctx *ctx) { return ctx ? ctx->launches : 0; }

int tc_ctx_set_t1_group(tc_ctx *ctx, int lanes)
{
    if (!ctx || (lanes != 8 && lanes != 16 && lanes != 32)) return TC_E_ARG;
    ctx->t1_group = lanes;
    return TC_OK;
}

int tc_ctx_t1_group(const tc_ctx *ctx) { return ctx ? ctx->t1_group : TC_E_ARG; }

int tc_ctx_set_dwt_variant(tc_ctx *ctx, int variant)
{
    if (!ctx || (variant != TC_DWT_CPASYNC && variant != TC_DWT_TMA)) return TC_E_ARG;
    ctx->dwt_variant = variant;
    return TC_OK;
}

int tc_ctx_dwt_variant(const tc_ctx *ctx) { return ctx ? ctx->dwt_variant : TC_E_ARG; }

void *tc_ctx_stream(const tc_ctx *ctx) { return ctx ? static_cast<void *>(ctx->stream) : nullptr; }

int tc_ctx_pool_bytes(tc_ctx *ctx, size_t *reserved)
{
    if (!ctx || !reserved) return TC_E_ARG;
    *reserved = 0;
    if (!ctx->pool) return TC_OK;
    uint64_t v = 0;
    const cudaError_t e = cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &v);
    if (e != cudaSuccess) return cuda_status(ctx, e, "tc_ctx_pool_bytes");
    *reserved = (size_t)v;
    return TC_OK;
}

int tc_ctx_trim(tc_ctx *ctx)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!ctx->pool) return TC_OK;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaMemPoolTrimTo(ctx->pool, 0);
    return cuda_status(ctx, e, "tc_ctx_trim");
}

int tc_t1_decode(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order, int n, const uint8_t *d_pool,
                 uint64_t pool_len, void *d_out, uint64_t out_elems, int out_mode, float recon_r, int max_bitplanes)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!d_desc || !d_out || (!d_pool && pool_len))) ||
        ((out_mode & ~TC_T1_STYLED) != TC_T1_OUT_DEQUANT && (out_mode & ~TC_T1_STYLED) != TC_T1_OUT_RAW) ||
        !(recon_r >= 0.0f && recon_r < 1.0f))
        return fail(ctx, TC_E_ARG, "tc_t1_decode: bad argument");
    if (max_bitplanes <= 0 || max_bitplanes > 31) max_bitplanes = 31;
    return cuda_status(ctx,
                       launch_t1_decode(ctx, d_desc, d_order, n, d_pool, pool_len, d_out, out_elems, out_mode,
                                        recon_r, max_bitplanes),
                       "tc_t1_decode");
}

int tc_t1_sort_order(const tc_cblk_desc *h_desc, int n, uint32_t *h_order)
{
    if (n < 0 || (n > 0 && (!h_desc || !h_order))) return TC_E_ARG;
    std::vector<std::pair<uint64_t, uint32_t>> key(n);
    for (int i = 0; i < n; i++) {
        const tc_cblk_desc &d = h_desc[i];
        const uint64_t work = (uint64_t)d.passes * d.w * d.h;
        key[i] = {(work << 24) | std::min<uint64_t>(d.seg_len, (1u << 24) - 1), (uint32_t)i};
    }
    std::stable_sort(key.begin(), key.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    for (int i = 0; i < n; i++) h_order[i] = key[i].second;
    return TC_OK;
}

int tc_dequantize_raw(tc_ctx *ctx, const tc_cblk_desc *d_desc, int n, const uint32_t *d_raw, void *d_out,
                      uint64_t elems, float recon_r)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!d_desc || !d_raw || !d_out)) || !(recon_r >= 0.0f && recon_r < 1.0f))
        return fail(ctx, TC_E_ARG, "tc_dequantize_raw: bad argument");
    return cuda_status(ctx, launch_dequant_raw(ctx, d_desc, n, d_raw, d_out, elems, recon_r), "tc_dequantize_raw");
}

static int dwt_args_ok(const void *in, int ip, const void *out, int op, int w, int h, int levels)
{
    return in && out && w > 0 && h > 0 && ip >= w && op >= w && levels >= 0 && levels <= 32;
}

static int dwt_forward(tc_ctx *ctx, int wavelet, int rounding, const void *d_in, int ip, void *d_out, int op, int w,
                       int h, int levels)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!dwt_args_ok(d_in, ip, d_out, op, w, h, levels) || d_in == d_out)
        return fail(ctx, TC_E_ARG, "forward DWT: bad argument");
    if (levels == 0) {
        cudaError_t e = cudaMemcpy2DAsync(d_out, (size_t)op * 4, d_in, (size_t)ip * 4, (size_t)w * 4, h,
                                          cudaMemcpyDeviceToDevice, ctx->stream);
        return cuda_status(ctx, e, "forward DWT copy");
    }
    // Level l reads the previous LL (the input for l = 1) and writes its LL
    // into a ping-pong scratch plane; the deepest LL lands in the output.
    std::vector<int> ws, hs;
    level_sizes(w, h, levels, ws, hs);
    const size_t slab = (size_t)ws[1] * hs[1] * 4;
    cudaError_t e = ctx->scratch.ensure(2 * slab);
    if (e != cudaSuccess) return cuda_status(ctx, e, "forward DWT scratch");
    const void *src = d_in;
    int sp = ip;
    for (int l = 1; l <= levels; l++) {
        LevelIO io{};
        io.w = ws[l - 1];
        io.h = hs[l - 1];
        io.ncomp = 1;
        io.ll[0] = src;
        io.ll_pitch = sp;
        io.bands[0] = d_out;
        io.bands_pitch = op;
        if (l == levels) {
            io.out[0] = d_out;
            io.out_pitch = op;
        } else {
            io.out[0] = static_cast<char *>(ctx->scratch.ptr) + ((l - 1) & 1) * slab;
            io.out_pitch = ws[1];
        }
        e = launch_fdwt_level(ctx, io, wavelet, rounding);
        if (e != cudaSuccess) return cuda_status(ctx, e, "forward DWT");
        src = io.out[0];
        sp = io.out_pitch;
    }
    return TC_OK;
}

static int dwt_reverse(tc_ctx *ctx, int wavelet, int rounding, const void *d_in, int ip, void *d_out, int op, int w,
                       int h, int levels)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!dwt_args_ok(d_in, ip, d_out, op, w, h, levels) || d_in == d_out)
        return fail(ctx, TC_E_ARG, "reverse DWT: bad argument");
    if (levels == 0) {
        cudaError_t e = cudaMemcpy2DAsync(d_out, (size_t)op * 4, d_in, (size_t)ip * 4, (size_t)w * 4, h,
                                          cudaMemcpyDeviceToDevice, ctx->stream);
        return cuda_status(ctx, e, "reverse DWT copy");
    }
    cudaError_t e = ctx->scratch.ensure(std::max<size_t>(reverse_scratch_bytes(w, h, levels, 1), 256));
    if (e != cudaSuccess) return cuda_status(ctx, e, "reverse DWT scratch");
    const void *in[1] = {d_in};
    void *out[1] = {d_out};
    return run_reverse(ctx, wavelet, rounding, in, ip, w, h, levels, 1, static_cast<char *>(ctx->scratch.ptr), out,
                       op, -1, 0, 0);
}

int tc_dwt_forward53(tc_ctx *ctx, const int32_t *d_in, int in_pitch, int32_t *d_out, int out_pitch, int w, int h,
                     int levels, int rounding)
{
    if (rounding != TC_ROUND_FLOOR && rounding != TC_ROUND_TRUNC) return fail(ctx, TC_E_ARG, "bad rounding");
    return dwt_forward(ctx, 0, rounding, d_in, in_pitch, d_out, out_pitch, w, h, levels);
}

int tc_dwt_forward97(tc_ctx *ctx, const float *d_in, int in_pitch, float *d_out, int out_pitch, int w, int h,
                     int levels)
{
    return dwt_forward(ctx, 1, 0, d_in, in_pitch, d_out, out_pitch, w, h, levels);
}

int tc_dwt_reverse53(tc_ctx *ctx, const int32_t *d_in, int in_pitch, int32_t *d_out, int out_pitch, int w, int h,
                     int levels, int rounding)
{
    if (rounding != TC_ROUND_FLOOR && rounding != TC_ROUND_TRUNC) return fail(ctx, TC_E_ARG, "bad rounding");
    return dwt_reverse(ctx, 0, rounding, d_in, in_pitch, d_out, out_pitch, w, h, levels);
}

int tc_dwt_reverse97(tc_ctx *ctx, const float *d_in, int in_pitch, float *d_out, int out_pitch, int w, int h,
                     int levels)
{
    return dwt_reverse(ctx, 1, 0, d_in, in_pitch, d_out, out_pitch, w, h, levels);
}

static int color_args_ok(int kind, int ncomp, const void *const *in, const void *const *out, int ip, int op, int w,
                         int h, int bits)
{
    if (kind < TC_COLOR_DC || kind > TC_COLOR_ICT || ncomp < 1 || ncomp > 4 || !in || !out) return 0;
    if ((kind != TC_COLOR_DC) && ncomp < 3) return 0;
    const int b = bits & ~TC_SIGNED;
    if (w <= 0 || h <= 0 || ip < w || op < w || b < 1 || b > 16) return 0;
    for (int c = 0; c < ncomp; c++)
        if (!in[c] || !out[c]) return 0;
    return 1;
}

int tc_color_inverse(tc_ctx *ctx, int kind, int ncomp, void *const *d_in, int in_type, int in_pitch,
                     void *const *d_out, int out_type, int out_pitch, int w, int h, int bits)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!color_args_ok(kind, ncomp, d_in, d_out, in_pitch, out_pitch, w, h, bits) ||
        (in_type != TC_INT32 && in_type != TC_FLOAT32) ||
        (out_type != TC_U8 && out_type != TC_U16 && out_type != TC_INT32) || (out_type == TC_U8 && bits > 8))
        return fail(ctx, TC_E_ARG, "tc_color_inverse: bad argument");
    return cuda_status(ctx,
                       launch_color_inverse(ctx, kind, ncomp, d_in, in_type, in_pitch, d_out, out_type, out_pitch,
                                            w, h, bits),
                       "tc_color_inverse");
}

int tc_color_forward(tc_ctx *ctx, int kind, int ncomp, const void *const *d_in, int in_type, int in_pitch,
                     void *const *d_out, int out_type, int out_pitch, int w, int h, int bits)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!color_args_ok(kind, ncomp, d_in, d_out, in_pitch, out_pitch, w, h, bits) ||
        (in_type != TC_U8 && in_type != TC_U16 && in_type != TC_INT32) ||
        (out_type != TC_INT32 && out_type != TC_FLOAT32))
        return fail(ctx, TC_E_ARG, "tc_color_forward: bad argument");
    return cuda_status(ctx,
                       launch_color_forward(ctx, kind, ncomp, d_in, in_type, in_pitch, d_out, out_type, out_pitch,
                                            w, h, bits),
                       "tc_color_forward");
}

int tc_j2k_read_header(const uint8_t *h_cs, size_t len, tc_image_info *info)
{
    if (!h_cs || !info || len < 2) return TC_E_ARG;
    std::string err;
    return read_header(h_cs, len, *info, err);
}

}  // extern "C"

// A parsed codestream handed out through the C ABI: the public struct first,
// then the owning parse result.
struct ParsedBox {
    tc_j2k_parsed pub;
    Parsed *own;
};

extern "C" {

int tc_j2k_parse(const uint8_t *h_cs, size_t len, tc_j2k_parsed **out)
{
    if (!h_cs || !out || len < 2) return TC_E_ARG;
    *out = nullptr;
    auto *holder = new (std::nothrow) Parsed;
    if (!holder) return TC_E_OOM;
    std::string err;
    const int rc = parse_codestream(h_cs, len, *holder, err);
    if (rc) {
        delete holder;
        return rc;
    }
    ParsedBox *b = new (std::nothrow) ParsedBox;
    if (!b) {
        delete holder;
        return TC_E_OOM;
    }
    std::memset(&b->pub, 0, sizeof b->pub);
    b->own = holder;
    b->pub.info = holder->info;
    b->pub.desc = holder->desc.data();
    b->pub.tiles = holder->tiles.data();
    b->pub.pool_is_cs = holder->pool_is_cs ? 1 : 0;
    b->pub.pool = holder->pool_is_cs ? h_cs : holder->own_pool.data();
    b->pub.pool_len = holder->pool_is_cs ? len : holder->own_pool.size();
    *out = &b->pub;
    return TC_OK;
}

void tc_j2k_parsed_free(tc_j2k_parsed *p)
{
    if (!p) return;
    ParsedBox *b = reinterpret_cast<ParsedBox *>(p);
    delete b->own;
    delete b;
}

int tc_plan_create(tc_ctx *ctx, const uint8_t *const *h_cs, const size_t *lens, int nimages, tc_plan **out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!h_cs || !lens || nimages < 1 || !out) return fail(ctx, TC_E_ARG, "tc_plan_create: bad argument");
    *out = nullptr;
    auto *P = new (std::nothrow) tc_plan;
    if (!P) return fail(ctx, TC_E_OOM, "tc_plan_create");
    rc = plan_build(ctx, h_cs, lens, nimages, P);
    if (rc) {
        tc_plan_destroy(P);
        return rc;
    }
    *out = P;
    return TC_OK;
}

int tc_plan_rebuild(tc_plan *P, const uint8_t *const *h_cs, const size_t *lens, int nimages)
{
    if (!P || !h_cs || !lens || nimages < 1) return TC_E_ARG;
    int rc = check_ctx(P->ctx);
    if (rc) return rc;
    // wait for the previous execute before its buffers are overwritten
    cudaError_t e = cudaStreamSynchronize(P->ctx->stream);
    if (e != cudaSuccess) return cuda_status(P->ctx, e, "tc_plan_rebuild");
    // cached graphs stay: they are keyed by their launch parameters, so a
    // batch of the same shape replays or updates one
    return plan_build(P->ctx, h_cs, lens, nimages, P);
}

int tc_plan_rebuild_parsed(tc_plan *P, const tc_j2k_parsed *const *parsed, int nimages)
{
    if (!P || !parsed || nimages < 1) return TC_E_ARG;
    int rc = check_ctx(P->ctx);
    if (rc) return rc;
    std::vector<const Parsed *> pp(nimages);
    std::vector<const uint8_t *> pools(nimages);
    std::vector<uint64_t> plens(nimages);
    for (int i = 0; i < nimages; i++) {
        if (!parsed[i]) return fail(P->ctx, TC_E_ARG, "tc_plan_rebuild_parsed: null image");
        const ParsedBox *b = reinterpret_cast<const ParsedBox *>(parsed[i]);
        pp[i] = b->own;
        pools[i] = b->pub.pool;
        plens[i] = b->pub.pool_len;
    }
    cudaError_t e = cudaStreamSynchronize(P->ctx->stream);
    if (e != cudaSuccess) return cuda_status(P->ctx, e, "tc_plan_rebuild_parsed");
    return plan_build_parsed(P->ctx, pp.data(), pools.data(), plens.data(), nimages, P);
}

int tc_plan_destroy(tc_plan *P)
{
    if (!P) return TC_E_ARG;
    if (P->ctx) {
        cudaSetDevice(P->ctx->device);
        cudaStreamSynchronize(P->ctx->stream);
    }
    P->pool.release();
    P->desc.release();
    P->order.release();
    P->coef.release();
    P->scratch.release();
    P->h_pool.release();
    P->h_desc.release();
    P->h_order.release();
    P->h_jobs.release();
    P->jobs.release();
    if (P->jobs_uploaded) cudaEventDestroy(P->jobs_uploaded);
    for (auto &e : P->ev)
        if (e) cudaEventDestroy(e);
    plan_drop_graphs(P);
    delete P;
    return TC_OK;
}

int tc_plan_set_profiling(tc_plan *P, int on)
{
    if (!P) return TC_E_ARG;
    int rc = check_ctx(P->ctx);
    if (rc) return rc;
    if (on && !P->ev[0])
        for (auto &e : P->ev) {
            cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) return cuda_status(P->ctx, r, "cudaEventCreate");
        }
    P->profiling = on != 0;
    return TC_OK;
}

int tc_plan_stage_ms(tc_plan *P, float *t1_ms, float *dwt_ms)
{
    if (!P || !P->profiling || !t1_ms || !dwt_ms) return TC_E_ARG;
    int rc = check_ctx(P->ctx);
    if (rc) return rc;
    cudaError_t e = cudaEventSynchronize(P->ev[2]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(t1_ms, P->ev[0], P->ev[1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(dwt_ms, P->ev[1], P->ev[2]);
    return cuda_status(P->ctx, e, "tc_plan_stage_ms");
}

int tc_plan_output_bytes(const tc_plan *P, int image, size_t *bytes)
{
    if (!P || !bytes || image < 0 || image >= (int)P->imgs.size()) return TC_E_ARG;
    *bytes = P->imgs[image].out_bytes;
    return TC_OK;
}

int tc_plan_image_info(const tc_plan *P, int image, tc_image_info *info)
{
    if (!P || !info || image < 0 || image >= (int)P->imgs.size()) return TC_E_ARG;
    *info = P->imgs[image].info;
    return TC_OK;
}

// The launch parameters of a graph-mode execute: equal keys mean the same
// kernels with the same arguments.  topo keeps only the launch topology.
static void plan_graph_key(const tc_plan *P, void *const *d_out, std::vector<uint64_t> &key,
                           std::vector<uint64_t> &topo)
{
    const int *cc = P->class_counts;
    topo = {(uint64_t)P->ctx->t1_group, (uint64_t)P->dwt_launches.size()};
    for (int k = 0; k < 6; k++) topo.push_back(cc[k] > 0);
    // the heavy queue and the 8-in-16 merge change the Tier-1 launches
    topo.push_back(cc[0] > 0 && cc[1] > 0 && cc[1] <= 148 && 8 * cc[1] <= cc[0]);
    topo.push_back(cc[0] > 0 && cc[1] > 0 && 2 * cc[0] <= cc[1]);
    topo.push_back(cc[3] > 0 && cc[4] > 0 && cc[4] <= 148 && 8 * cc[4] <= cc[3]);
    for (const tc_plan::DwtLaunch &L : P->dwt_launches)
        for (int v : {L.wavelet, L.color, L.ncomp, L.otype, L.bits}) topo.push_back((uint64_t)(int64_t)v);
    key = topo;
    uint32_t rbits;
    std::memcpy(&rbits, &P->recon_r, 4);
    for (uint64_t v : {(uint64_t)P->ncblk, (uint64_t)(uintptr_t)P->pool.ptr, (uint64_t)P->pool.size,
                       (uint64_t)(uintptr_t)P->desc.ptr, (uint64_t)(uintptr_t)P->order.ptr,
                       (uint64_t)(uintptr_t)P->coef.ptr, (uint64_t)(uintptr_t)P->scratch.ptr,
                       (uint64_t)(uintptr_t)P->jobs.ptr, (uint64_t)rbits})
        key.push_back(v);
    for (int k = 0; k < 6; k++) key.push_back((uint64_t)cc[k]);
    for (const tc_plan::DwtLaunch &L : P->dwt_launches)
        for (int v : {L.first, L.njobs, L.ntiles}) key.push_back((uint64_t)v);
    // images without a transform take their colour launch's pointers as
    // parameters
    for (size_t i = 0; i < P->imgs.size(); i++)
        if (P->imgs[i].info.levels == 0) {
            key.push_back((uint64_t)(uintptr_t)d_out[i]);
            key.push_back(P->imgs[i].coef_off);
            topo.push_back(i);
        }
}

// Captures one execute's launches on the context's capture stream (the
// caller's stream may be the legacy default stream, which cannot be
// captured); the graph is launched on the caller's stream.
static int plan_capture(tc_plan *P, void *const *d_out, cudaGraph_t *g, uint64_t *launches)
{
    tc_ctx *ctx = P->ctx;
    cudaError_t e = ensure_side_streams(ctx);
    if (e != cudaSuccess) return cuda_status(ctx, e, "graph capture");
    const uint64_t l0 = ctx->launches;
    cudaStream_t caller = ctx->stream;
    ctx->stream = ctx->capture;
    e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        ctx->stream = caller;
        return cuda_status(ctx, e, "graph capture");
    }
    const int rc = plan_run(P, d_out, true);
    e = cudaStreamEndCapture(ctx->stream, g);
    ctx->stream = caller;
    *launches = ctx->launches - l0;
    ctx->launches = l0;
    if (rc) {
        if (*g) cudaGraphDestroy(*g);
        *g = nullptr;
        return rc;
    }
    return cuda_status(ctx, e, "graph capture");
}

int tc_plan_execute(tc_plan *P, void *const *d_out)
{
    if (!P || !d_out) return TC_E_ARG;
    int rc = check_ctx(P->ctx);
    if (rc) return rc;
    for (size_t i = 0; i < P->imgs.size(); i++)
        if (!d_out[i]) return fail(P->ctx, TC_E_ARG, "tc_plan_execute: null output");
    if (!P->use_graph || P->profiling) return plan_run(P, d_out);
    tc_ctx *ctx = P->ctx;
    // the DWT job table for these outputs, uploaded outside any graph
    if ((rc = run_reverse_batched(P, d_out, false))) return rc;
    std::vector<uint64_t> key, topo;
    plan_graph_key(P, d_out, key, topo);
    tc_plan::Graph *hit = nullptr, *same_topo = nullptr;
    for (tc_plan::Graph &g : P->graphs) {
        if (g.key == key) hit = &g;
        else if (g.topo == topo && !same_topo) same_topo = &g;
    }
    cudaError_t e;
    if (!hit && same_topo) {
        // same shape bucket: update the cached graph's parameters in place
        cudaGraph_t g = nullptr;
        uint64_t nl = 0;
        if ((rc = plan_capture(P, d_out, &g, &nl))) return rc;
        cudaGraphExecUpdateResultInfo info{};
        e = cudaGraphExecUpdate(same_topo->exec, g, &info);
        cudaGraphDestroy(g);
        if (e == cudaSuccess) {
            same_topo->key = key;
            same_topo->launches = nl;
            hit = same_topo;
            P->graph_updates++;
        } else {
            cudaGetLastError();  // an update refused is not an error: instantiate instead
        }
    }
    if (!hit) {
        // A new bucket: run normally first (kernel attributes, side streams
        // and the context's one-time set-up), then capture the same work.
        if ((rc = plan_run(P, d_out, true))) return rc;
        cudaGraph_t g = nullptr;
        uint64_t nl = 0;
        if ((rc = plan_capture(P, d_out, &g, &nl))) return rc;
        tc_plan::Graph G;
        e = cudaGraphInstantiate(&G.exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_status(ctx, e, "graph instantiate");
        G.key = key;
        G.topo = topo;
        G.launches = nl;
        G.last_use = ++P->graph_tick;
        if (P->graphs.size() >= kMaxGraphs) {
            auto lru = std::min_element(P->graphs.begin(), P->graphs.end(),
                                        [](const tc_plan::Graph &a, const tc_plan::Graph &b) {
                                            return a.last_use < b.last_use;
                                        });
            cudaGraphExecDestroy(lru->exec);
            P->graphs.erase(lru);
        }
        P->graphs.push_back(G);
        P->graph_captures++;
        return TC_OK;
    }
    hit->last_use = ++P->graph_tick;
    e = cudaGraphLaunch(hit->exec, ctx->stream);
    if (e != cudaSuccess) return cuda_status(ctx, e, "graph launch");
    ctx->launches += hit->launches;
    P->graph_replays++;
    return TC_OK;
}

int tc_plan_device_bytes(const tc_plan *P, size_t *bytes)
{
    if (!P || !bytes) return TC_E_ARG;
    *bytes = P->pool.size + P->desc.size + P->order.size + P->coef.size + P->scratch.size + P->jobs.size;
    return TC_OK;
}

int tc_plan_graph_stats(const tc_plan *P, uint64_t *captures, uint64_t *updates, uint64_t *replays)
{
    if (!P || !captures || !updates || !replays) return TC_E_ARG;
    *captures = P->graph_captures;
    *updates = P->graph_updates;
    *replays = P->graph_replays;
    return TC_OK;
}

int tc_plan_set_graph(tc_plan *P, int on)
{
    if (!P) return TC_E_ARG;
    P->use_graph = on != 0;
    if (!on) plan_drop_graphs(P);
    return TC_OK;
}

int tc_decode_j2k(tc_ctx *ctx, const uint8_t *h_cs, size_t len, void *h_out, size_t out_bytes, tc_image_info *info)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!h_cs || !len || !h_out) return fail(ctx, TC_E_ARG, "tc_decode_j2k: bad argument");
    // The plan borrows the context's grow-only buffers, so repeated decodes
    // of similar images allocate nothing after the first call.
    tc_plan P;
    P.pool = ctx->tmp_pool;
    P.desc = ctx->tmp_desc;
    P.order = ctx->tmp_order;
    P.coef = ctx->tmp_coef;
    P.scratch = ctx->scratch;
    P.h_pool = ctx->stage_pool;
    P.h_desc = ctx->stage_desc;
    P.h_order = ctx->stage_order;
    P.jobs = ctx->tmp_jobs;
    P.h_jobs = ctx->stage_jobs;
    P.jobs_uploaded = ctx->jobs_uploaded;
    auto give_back = [&]() {
        ctx->tmp_pool = P.pool;
        ctx->tmp_desc = P.desc;
        ctx->tmp_order = P.order;
        ctx->tmp_coef = P.coef;
        ctx->scratch = P.scratch;
        ctx->stage_pool = P.h_pool;
        ctx->stage_desc = P.h_desc;
        ctx->stage_order = P.h_order;
        ctx->tmp_jobs = P.jobs;
        ctx->stage_jobs = P.h_jobs;
        ctx->jobs_uploaded = P.jobs_uploaded;
    };
    // A codestream in pinned memory is uploaded while it is parsed: the
    // segment pool of a single-layer stream is the codestream itself (the
    // plan re-uploads a gathered pool over it otherwise, in stream order).
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, h_cs) == cudaSuccess && pa.type == cudaMemoryTypeHost) {
        cudaMemPool_t mp = nullptr;
        const size_t bytes = (len + 15) & ~size_t(15);  // the plan's pool size for this stream
        cudaError_t e = ctx_mem_pool(ctx, &mp);
        if (e == cudaSuccess) e = P.pool.ensure_on(bytes, ctx->stream, mp);
        if (e == cudaSuccess) e = cudaMemcpyAsync(P.pool.ptr, h_cs, len, cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) {
            give_back();
            return cuda_status(ctx, e, "tc_decode_j2k upload");
        }
        P.preloaded = h_cs;
        P.preloaded_len = len;
    } else {
        cudaGetLastError();  // pageable memory: not an error
    }
    const uint8_t *cs[1] = {h_cs};
    size_t lens[1] = {len};
    rc = plan_build(ctx, cs, lens, 1, &P);
    if (rc) {
        give_back();
        return rc;
    }
    const size_t need = P.imgs[0].out_bytes;
    if (info) *info = P.imgs[0].info;
    if (out_bytes < need) {
        give_back();
        return fail(ctx, TC_E_ARG, "tc_decode_j2k: output buffer too small");
    }
    cudaError_t e = ctx->tmp_out.ensure(need);
    if (e != cudaSuccess) {
        give_back();
        return cuda_status(ctx, e, "tc_decode_j2k output");
    }
    void *outs[1] = {ctx->tmp_out.ptr};
    rc = plan_run(&P, outs);
    give_back();
    if (rc) return rc;
    e = cudaMemcpyAsync(h_out, ctx->tmp_out.ptr, need, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_status(ctx, e, "tc_decode_j2k D2H");
    return tc_ctx_synchronize(ctx);
}

int tc_decode_j2k_file(tc_ctx *ctx, const char *path, void *h_out, size_t out_bytes, tc_image_info *info)
{
    if (!path) return TC_E_ARG;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(ctx, TC_E_NOFILE, std::string("cannot open ") + path);
    std::vector<uint8_t> buf;
    uint8_t tmp[1 << 16];
    size_t k;
    while ((k = std::fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + k);
    std::fclose(f);
    return tc_decode_j2k(ctx, buf.data(), buf.size(), h_out, out_bytes, info);
}

int tc_encode_j2k(const tc_encode_params *p, const void *h_planes, uint8_t *h_out, size_t cap, size_t *out_len)
{
    if (!p || !h_planes || !out_len) return TC_E_ARG;
    std::vector<uint8_t> cs;
    std::string err;
    const int rc = encode_codestream(*p, h_planes, cs, err);
    if (rc) return rc;
    *out_len = cs.size();
    if (!h_out || cap < cs.size()) return TC_E_ARG;
    std::memcpy(h_out, cs.data(), cs.size());
    return TC_OK;
}

int tc_encode_j2k_gpu(tc_ctx *ctx, const tc_encode_params *p, const void *h_planes, uint8_t *h_out, size_t cap,
                      size_t *out_len)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!p || !h_planes || !out_len) return fail(ctx, TC_E_ARG, "tc_encode_j2k_gpu: bad argument");
    std::string err;
    EncodeLayout L;
    if ((rc = encode_layout(*p, L, err))) return fail(ctx, rc, err);
    for (int c = 0; c < p->ncomp; c++)
        if (L.dx[c] != 1 || L.dy[c] != 1)
            return fail(ctx, TC_E_UNSUPPORTED, "tc_encode_j2k_gpu: subsampled components (use tc_encode_j2k)");
    if (p->cblk_style)
        return fail(ctx, TC_E_UNSUPPORTED, "tc_encode_j2k_gpu: code-block style modes (use tc_encode_j2k)");
    if (p->roi_x1 > p->roi_x0 || p->roi_y1 > p->roi_y0)
        return fail(ctx, TC_E_UNSUPPORTED, "tc_encode_j2k_gpu: region of interest (use tc_encode_j2k)");
    const int W = p->width, H = p->height, C = p->ncomp, B = p->bits, NL = p->levels;
    const size_t np = (size_t)W * H;
    const int sb = B <= 8 ? 1 : 2;
    const bool rev = p->reversible != 0;
    const int nb = (int)L.jobs.size();
    // worst case per block: about 1.2 decisions per sample per bit-plane over
    // 31 bit-planes, at most one bit per decision, plus the termination
    uint32_t bcap = 0;
    for (int c = 0; c < C; c++) bcap = std::max<uint32_t>(bcap, 5u << (2 * L.cblk[c]));
    bcap += 256;
    DevBuf &in = ctx->enc[0], &col = ctx->enc[1], &coef = ctx->enc[2], &desc = ctx->enc[3], &words = ctx->enc[4],
           &res = ctx->enc[5], &off = ctx->enc[6], &packed = ctx->enc[7];
    auto done = [&](int status) {
        cudaStreamSynchronize(ctx->stream);
        return status;
    };
    cudaError_t e;
    if ((e = in.ensure(np * C * sb)) != cudaSuccess || (e = col.ensure(np * C * 4)) != cudaSuccess ||
        (e = coef.ensure(np * C * 4)) != cudaSuccess ||
        (e = desc.ensure(std::max(1, nb) * sizeof(tc_t1_enc_desc))) != cudaSuccess ||
        (e = words.ensure((size_t)std::max(1, nb) * bcap)) != cudaSuccess ||
        (e = res.ensure(std::max(1, nb) * sizeof(tc_t1_enc_result))) != cudaSuccess ||
        (e = off.ensure(std::max(1, nb) * sizeof(uint64_t))) != cudaSuccess)
        return done(cuda_status(ctx, e, "tc_encode_j2k_gpu allocation"));
    if ((e = cudaMemcpyAsync(in.ptr, h_planes, np * C * sb, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
        return done(cuda_status(ctx, e, "tc_encode_j2k_gpu upload"));
    // forward colour transform with the DC shift (ISO G.1-G.2), per plane the DWT (ISO F.4)
    const void *ip[4];
    void *cp[4];
    for (int c = 0; c < C; c++) {
        ip[c] = static_cast<char *>(in.ptr) + c * np * sb;
        cp[c] = static_cast<char *>(col.ptr) + c * np * 4;
    }
    const int kind = p->mct && C >= 3 ? (rev ? TC_COLOR_RCT : TC_COLOR_ICT) : TC_COLOR_DC;
    e = launch_color_forward(ctx, kind, C, ip, sb == 1 ? TC_U8 : TC_U16, W, cp, rev ? TC_INT32 : TC_FLOAT32, W, W, H,
                             B | (p->is_signed ? TC_SIGNED : 0));
    if (e != cudaSuccess) return done(cuda_status(ctx, e, "tc_encode_j2k_gpu colour"));
    for (int c = 0; c < C; c++) {
        rc = dwt_forward(ctx, rev ? 0 : 1, TC_ROUND_FLOOR, cp[c], W, static_cast<char *>(coef.ptr) + c * np * 4, W,
                         W, H, NL);
        if (rc) return done(rc);
    }
    // Tier-1 of every block with Mb = 31 (the codeword does not depend on Mb)
    std::vector<tc_t1_enc_desc> hd(nb);
    for (int k = 0; k < nb; k++) {
        const EncodeLayout::Job &jb = L.jobs[k];
        const Band &b = L.geo[jb.c][jb.r].bands[jb.bi];
        const int cx = jb.i << b.cbw_log2, cy = jb.j << b.cbh_log2;
        tc_t1_enc_desc &d = hd[k];
        std::memset(&d, 0, sizeof d);
        d.in_off = (uint64_t)jb.c * np + (uint64_t)(b.y0 + cy) * W + (uint64_t)(b.x0 + cx);
        d.in_pitch = (uint32_t)W;
        d.w = (uint16_t)std::min(1 << b.cbw_log2, b.w - cx);
        d.h = (uint16_t)std::min(1 << b.cbh_log2, b.h - cy);
        d.orient = (uint8_t)b.orient;
        d.mb = 31;
        d.flags = rev ? 0 : TC_CBLK_IRREVERSIBLE;
        d.inv_step = rev ? 1.0f : 1.0f / b.step;
    }
    std::vector<tc_t1_enc_result> hr(nb);
    if ((e = cudaMemcpyAsync(desc.ptr, hd.data(), nb * sizeof(tc_t1_enc_desc), cudaMemcpyHostToDevice, ctx->stream)) !=
            cudaSuccess ||
        (e = launch_t1_encode(ctx, static_cast<tc_t1_enc_desc *>(desc.ptr), nb, coef.ptr,
                              static_cast<uint8_t *>(words.ptr), bcap, static_cast<tc_t1_enc_result *>(res.ptr))) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(hr.data(), res.ptr, nb * sizeof(tc_t1_enc_result), cudaMemcpyDeviceToHost,
                             ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return done(cuda_status(ctx, e, "tc_encode_j2k_gpu Tier-1"));
    // pack the codewords and bring them back
    std::vector<uint64_t> ho(nb);
    uint64_t total = 0;
    for (int k = 0; k < nb; k++) {
        if (hr[k].status) return done(fail(ctx, TC_E_ARG, "tc_encode_j2k_gpu: code-block " + std::to_string(k) +
                                                              " status " + std::to_string(hr[k].status)));
        ho[k] = total;
        total += hr[k].len;
    }
    if ((e = ctx->enc_host.ensure(std::max<uint64_t>(total, 1))) != cudaSuccess)
        return done(cuda_status(ctx, e, "tc_encode_j2k_gpu staging"));
    uint8_t *hw = static_cast<uint8_t *>(ctx->enc_host.ptr);
    if ((e = packed.ensure(std::max<uint64_t>(total, 1))) != cudaSuccess ||
        (e = cudaMemcpyAsync(off.ptr, ho.data(), nb * sizeof(uint64_t), cudaMemcpyHostToDevice, ctx->stream)) !=
            cudaSuccess ||
        (e = launch_gather_codewords(ctx, static_cast<uint8_t *>(words.ptr), bcap,
                                     static_cast<tc_t1_enc_result *>(res.ptr), static_cast<uint64_t *>(off.ptr), nb,
                                     static_cast<uint8_t *>(packed.ptr))) != cudaSuccess ||
        (e = cudaMemcpyAsync(hw, packed.ptr, total, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
        return done(cuda_status(ctx, e, "tc_encode_j2k_gpu read-back"));
    std::vector<CodedBlock> coded(nb);
    for (int k = 0; k < nb; k++) {
        coded[k].data = hw + ho[k];
        coded[k].len = hr[k].len;
        coded[k].passes = (int)hr[k].passes;
        coded[k].numbps = 31 - (int)hr[k].zero_bitplanes;
    }
    std::vector<uint8_t> cs;
    if ((rc = encode_assemble(*p, L, coded, cs, err))) return done(fail(ctx, rc, err));
    *out_len = cs.size();
    if (!h_out || cap < cs.size()) return done(fail(ctx, TC_E_ARG, "tc_encode_j2k_gpu: output buffer too small"));
    std::memcpy(h_out, cs.data(), cs.size());
    return done(TC_OK);
}

int tc_t1_encode(tc_ctx *ctx, const tc_t1_enc_desc *d_desc, int n, const void *d_in, uint8_t *d_out, uint32_t cap,
                 tc_t1_enc_result *d_res)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!d_desc || !d_in || !d_out || !d_res || cap == 0)))
        return fail(ctx, TC_E_ARG, "tc_t1_encode: bad argument");
    return cuda_status(ctx, launch_t1_encode(ctx, d_desc, n, d_in, d_out, cap, d_res), "tc_t1_encode");
}

int tc_t1_encode_block(const int32_t *h_coef, int w, int h, int orient, int mb, int passes, uint8_t *h_out, int cap,
                       int *len, int *passes_out, int *zero_bitplanes)
{
    if (!h_coef || !len || !passes_out || !zero_bitplanes) return TC_E_ARG;
    std::vector<uint8_t> out;
    const int rc = t1_encode_block(h_coef, w, h, orient, mb, passes, out, passes_out, zero_bitplanes);
    if (rc) return rc;
    *len = (int)out.size();
    if ((int)out.size() > cap || (!h_out && !out.empty())) return TC_E_ARG;
    if (!out.empty()) std::memcpy(h_out, out.data(), out.size());
    return TC_OK;
}

}  // extern "C"
