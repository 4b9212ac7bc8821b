/*
 * tc_j2k.h -- C ABI of the B200 (sm_100a) JPEG 2000 decode pipeline.
 *
 * This is the drop-in boundary for kgmoore/ThousandthChicken's device stages.
 * Each entry point names the reference interface it replaces (paths relative
 * to the reference project's ThousandthChicken/ directory).  Plain pointers
 * and sizes only: no C++ or framework types cross this boundary, and no C++
 * exception escapes it.
 *
 * Conventions
 *  - Status codes: TC_OK (0) or a negative TC_E_* value.  They replace the
 *    reference's tDeviceRC/cl_int (platform.h:9-11) and its thrown Error
 *    objects (basic.h:95-104).
 *  - A tc_ctx is bound to one CUDA device and one CUDA stream; every call on
 *    a ctx is stream-ordered on that stream.  A ctx may be used from one host
 *    thread at a time; distinct contexts are independent (no global mutable
 *    state apart from the read-only tables each kernel builds for itself).
 *  - Pointers named d_* are device pointers; h_* are host pointers.
 *  - Geometry: tile origin at (0,0); Mallat layout means the multi-level
 *    subbands sit in place in one plane (LL_N top-left; at each level the HL
 *    band right of LL, LH below it, HH diagonal).
 */
#ifndef TC_J2K_H
#define TC_J2K_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define TC_OK              0
#define TC_E_ARG          -1  /* invalid argument */
#define TC_E_OOM          -2  /* host or device allocation failed */
#define TC_E_CODESTREAM   -3  /* malformed codestream or code-block data */
#define TC_E_DEVICE       -4  /* CUDA error */
#define TC_E_TIMEOUT      -5  /* a bounded device wait gave up */
#define TC_E_UNSUPPORTED  -6  /* valid JPEG 2000 outside the supported subset */
#define TC_E_NOFILE       -7  /* file missing (Decoder.cpp:103-107 returns -2) */

/* ---- sample types -------------------------------------------------------- */
#define TC_U8     1
#define TC_U16    2
#define TC_INT32  3
#define TC_FLOAT32 4

/* ---- context ------------------------------------------------------------- */
typedef struct tc_ctx tc_ctx;

/* Create a context on `device` that issues work on `cuda_stream` (a
 * cudaStream_t; NULL = the legacy default stream).  Replaces the OpenCL
 * set-up of InitOpenCL (ocl_util.cpp:425-466) and KernelInitInfoBase
 * (platform.h:21-34). */
int tc_ctx_create(int device, void *cuda_stream, tc_ctx **out);
int tc_ctx_destroy(tc_ctx *ctx);
/* Wait for all work on the ctx's stream, then read and clear the device
 * error word; returns TC_E_CODESTREAM when a kernel flagged bad block data. */
int tc_ctx_synchronize(tc_ctx *ctx);
/* Message for the last failing call on this ctx ("" if none). */
const char *tc_ctx_last_error(const tc_ctx *ctx);
const char *tc_status_string(int status);
/* Library version: major*10000 + minor*100 + patch. */
int tc_version(void);
/* Number of kernel launches this ctx issued since creation (diagnostics). */
uint64_t tc_ctx_launch_count(const tc_ctx *ctx);
/* Lanes per code-block in the Tier-1 kernel: 32 (one warp per block), 16 or
 * 8 (two or four blocks per warp, decoded in lock-step).  The best width
 * depends on the block mix; the package's autotuner measures it per workload
 * and caches the choice.  Default 32. */
int tc_ctx_set_t1_group(tc_ctx *ctx, int lanes);
int tc_ctx_t1_group(const tc_ctx *ctx);
/* How the fused last reverse 9/7 level of three-component images stages
 * its subband tiles: TC_DWT_TMA (default) with 2-D tensor copies (TMA) on
 * an mbarrier, where the level's band width, row pitches and addresses are
 * multiples of 16 bytes (others fall back), or TC_DWT_CPASYNC with one
 * 4-byte asynchronous copy per sample.  Same results either way; the
 * package's autotuner times both per shape bucket. */
#define TC_DWT_CPASYNC 0
#define TC_DWT_TMA     1
int tc_ctx_set_dwt_variant(tc_ctx *ctx, int variant);
int tc_ctx_dwt_variant(const tc_ctx *ctx);
/* The CUDA stream (cudaStream_t) the ctx issues its work on. */
void *tc_ctx_stream(const tc_ctx *ctx);
/* Device memory the ctx's memory pool reserves now: the buffers of its
 * plans plus freed blocks the pool keeps mapped for regrowth.  A serving
 * loop admits work against it.  No counterpart in the reference. */
int tc_ctx_pool_bytes(tc_ctx *ctx, size_t *reserved);
/* Wait for the ctx's stream, then return the pool's unused blocks to the
 * device (after a plan is destroyed, its memory leaves the pool). */
int tc_ctx_trim(tc_ctx *ctx);

/* ---- Tier-1 code-block decode (CoefficientCoder) ------------------------- */

/* One code-block as Tier-2 leaves it.  Filled by the parser below, or by a
 * caller's own parser from the reference's type_codeblock in its
 * codeBlockCallback (codestream.h:12-14, codestream.c:465-466; fields from
 * codestream_image_types.h:30-120 and CodeBlockAdditionalInfo,
 * coefficientcoder_common.h:5-24). */
typedef struct tc_cblk_desc {
    uint64_t seg_off;        /* byte offset of the block's codeword in the pool;
                                with style BYPASS or TERMALL, of a 4-byte aligned
                                table of its codeword segments' lengths (uint32,
                                little-endian, one per segment the passes span)
                                that the codeword follows */
    uint64_t out_off;        /* element offset (4-byte elements) of sample (0,0) */
    uint32_t seg_len;        /* codeword bytes (cblk->length), table excluded */
    uint32_t out_pitch;      /* output row pitch in elements */
    float    step;           /* dequantisation step, irreversible blocks only */
    uint16_t w, h;           /* block size, 1..64 each */
    uint8_t  passes;         /* coding passes included (cblk->num_coding_passes) */
    uint8_t  mb;             /* magnitude bit-planes Mb of the subband (1..31) */
    uint8_t  zero_bitplanes; /* Mb - significant_bits */
    uint8_t  orient;         /* 0 LL, 1 HL, 2 LH, 3 HH (type_orient) */
    uint8_t  flags;          /* TC_CBLK_* */
    uint8_t  style;          /* code-block style, TC_CBLK_STYLE_* (0: none) */
    uint8_t  roi_shift;      /* ROI maxshift s (RGN, ISO Annex H; 0: none): mb
                                counts the s extra bit-planes, and a decoded
                                magnitude >= 2^s is shifted down by s */
    uint8_t  reserved[1];
} tc_cblk_desc;

#define TC_CBLK_IRREVERSIBLE 0x01  /* float output, multiply by step */

/* Code-block style bits (COD / COC SPcod, ISO Table A.19). */
#define TC_CBLK_STYLE_BYPASS  0x01  /* selective arithmetic coding bypass */
#define TC_CBLK_STYLE_RESET   0x02  /* contexts reset after each pass */
#define TC_CBLK_STYLE_TERMALL 0x04  /* every pass terminated */
#define TC_CBLK_STYLE_VSC     0x08  /* vertically stripe-causal contexts */
#define TC_CBLK_STYLE_PTERM   0x10  /* predictable termination */
#define TC_CBLK_STYLE_SEGSYM  0x20  /* segmentation symbols */

/* Output modes of tc_t1_decode. */
#define TC_T1_OUT_DEQUANT 0  /* int32 (reversible) or float (irreversible) values */
#define TC_T1_OUT_RAW     1  /* uint32 sign-magnitude, sign at bit 31, magnitude
                                bit b at bit b+31-Mb: the reference g_decode
                                output (coefficient_coder.cl:605-626,805-816) */

/* Or-ed into out_mode: the descriptors may carry code-block styles
 * (tc_cblk_desc.style); every block is decoded by the style-capable kernel.
 * Without it a block with a style that changes decoding is reported as an
 * error by tc_ctx_synchronize and left undecoded. */
#define TC_T1_STYLED      0x10

/* Decode n code-blocks in one persistent launch (one warp per code-block,
 * blocks taken from a device work queue in the order d_order gives; NULL =
 * descriptor order; the host-side tc_t1_sort_order() produces a
 * longest-first order).  With TC_T1_OUT_DEQUANT the inverse quantiser is
 * fused in: reconstruction point recon_r in [0,1) (ISO E.1.1.2; the
 * irreversible path adds it on the last decoded plane, the reversible path
 * only for truncated blocks; 0 = truncated value).  max_bitplanes bounds
 * Mb - zero_bitplanes over the blocks (0 = up to 31); it sizes the
 * magnitude storage, and a block above it is flagged as out of range.
 * d_out holds out_elems 4-byte elements: a block whose last sample,
 * out_off + (h-1)*out_pitch + w - 1, is not below out_elems is skipped before
 * anything is written and reported by tc_ctx_synchronize (the reference
 * trusts d_coefficientsOffset, coefficientcoder_common.h:5-24).
 * Replaces CoefficientCoder::decode_tile/decodeInit/decode
 * (CoefficientCoder.cpp:62-252) plus Quantizer::dequantize_tile
 * (Quantizer.cpp:181-216). */
int tc_t1_decode(tc_ctx *ctx, const tc_cblk_desc *d_desc, const uint32_t *d_order,
                 int n, const uint8_t *d_pool, uint64_t pool_len, void *d_out,
                 uint64_t out_elems, int out_mode, float recon_r, int max_bitplanes);

/* Host helper: write into h_order a permutation of 0..n-1 sorted by
 * decreasing estimated work (passes x area, then codeword length). */
int tc_t1_sort_order(const tc_cblk_desc *h_desc, int n, uint32_t *h_order);

/* Standalone inverse quantiser over TC_T1_OUT_RAW output: reads the raw word
 * of every block sample at the descriptor's out_off/out_pitch in d_raw and
 * writes int32 or float at the same place in d_out.  The number of decoded
 * bit-planes is taken from the pass count.  Replaces Quantizer::dequantization
 * and the subband_dequantization_lossless/lossy kernels
 * (Quantizer.cpp:126-175, quantizer_*_inverse.cl:16-44), with the sign
 * handled (defect D4 fixed).  d_raw and d_out each hold `elems` elements;
 * blocks placed beyond them are skipped and reported, as in tc_t1_decode. */
int tc_dequantize_raw(tc_ctx *ctx, const tc_cblk_desc *d_desc, int n,
                      const uint32_t *d_raw, void *d_out, uint64_t elems, float recon_r);

/* ---- DWT (DWTForward53/97, DWTReverse53/97, DWTKernel<T>::run) ----------- */

#define TC_ROUND_FLOOR 0  /* ISO F.3/F.4 floor lifting (conformant) */
#define TC_ROUND_TRUNC 1  /* C truncating division, as the reference kernels
                             (dwt_transform_buffer.cl:124-269) */

/* Multi-level forward transform of a w x h plane into Mallat layout.
 * Replaces DWTForward53::dwt / DWTForward97::dwt (DWTForward53.cpp:20-43,
 * DWTForward97.cpp:20-43) and DWTKernel<T>::run(in, out, sx, sy, levels)
 * (DWTKernel.cpp:158-178).  d_in is not modified. */
int tc_dwt_forward53(tc_ctx *ctx, const int32_t *d_in, int in_pitch,
                     int32_t *d_out, int out_pitch, int w, int h, int levels,
                     int rounding);
int tc_dwt_forward97(tc_ctx *ctx, const float *d_in, int in_pitch,
                     float *d_out, int out_pitch, int w, int h, int levels);

/* Multi-level reverse transform from Mallat layout back to samples.
 * Replaces DWTReverse53::dwt / DWTReverse97::dwt (DWTReverse53.cpp:23-43,
 * DWTReverse97.cpp:24-44) and DWT::iwt (DWT.cpp:57-114).  d_in is not
 * modified; d_out must not alias d_in. */
int tc_dwt_reverse53(tc_ctx *ctx, const int32_t *d_in, int in_pitch,
                     int32_t *d_out, int out_pitch, int w, int h, int levels,
                     int rounding);
int tc_dwt_reverse97(tc_ctx *ctx, const float *d_in, int in_pitch,
                     float *d_out, int out_pitch, int w, int h, int levels);

/* Allocation-free reverse 9/7 for callers that cannot allocate device
 * memory (code under stream capture that must not allocate, hosts whose
 * memory manager owns every device allocation, real-time paths that cannot
 * afford cudaMalloc/cudaFree).  No counterpart in the reference: its DWT
 * allocates and zero-fills a fresh output on every call (DWT.cpp:79-84).
 * Same transform and result as tc_dwt_reverse97, but it takes a CUDA stream
 * instead of a context, and the intermediate plane lives in a file-scope
 * device array of TC_DWT97_STATIC_SCRATCH_ELEMS floats (16 MiB) that every
 * GPU loading this library holds until exit.  Returns TC_E_ARG when
 * ceil(w/2) * ceil(h/2) exceeds that size (levels >= 2).  It calls no
 * cudaMalloc, cudaFree or allocating library routine.  Its first call on a
 * device looks up the array's address there (cudaGetSymbolAddress with that
 * device current, whatever the level count); make that first call before any
 * stream capture.  The address is cached for the process: do not call this
 * on a device after cudaDeviceReset on it.  Calls
 * share the array: calls whose work overlaps on the GPU race on it.  The
 * array keeps the last call's contents and nothing in it needs to start at
 * zero. */
#define TC_DWT97_STATIC_SCRATCH_ELEMS (4u * 1024u * 1024u)
int tc_dwt_reverse97_static(const float *d_in, int in_pitch, float *d_out, int out_pitch,
                            int w, int h, int levels, void *cuda_stream);

/* ---- colour transform + DC level shift (Preprocessor) -------------------- */

#define TC_COLOR_DC  0  /* DC level shift only, per component */
#define TC_COLOR_RCT 1  /* reversible component transform (components 0-2) */
#define TC_COLOR_ICT 2  /* irreversible component transform (components 0-2) */
/* Flag or-ed into a `bits` argument: the samples are signed (two's
 * complement, no DC level shift, clamped to [-2^(bits-1), 2^(bits-1)-1]). */
#define TC_SIGNED 0x100

/* Inverse: planes of in_type (TC_INT32 or TC_FLOAT32) -> inverse colour
 * transform, DC shift, rounding (float input: to nearest even) and clamp to
 * [0, 2^bits-1] -> planes of out_type (TC_U8, TC_U16 or TC_INT32).  With
 * bits | TC_SIGNED: no DC shift, clamp to the signed range, two's
 * complement in the same sample types.
 * Replaces Preprocessor::color_decoder_lossless/color_decoder_lossy/
 * idc_level_shifting (Preprocessor.cpp:44-180) and the tcr_kernel,
 * tci_kernel and idc_level_shift_kernel kernels; the ICT uses the ISO G.2
 * inverse (defect D9 fixed) and the dispatch follows the transform asked for
 * (defects D7/D8 fixed). */
int tc_color_inverse(tc_ctx *ctx, int kind, int ncomp,
                     void *const *d_in, int in_type, int in_pitch,
                     void *const *d_out, int out_type, int out_pitch,
                     int w, int h, int bits);

/* Forward: unsigned samples of in_type (TC_U8, TC_U16 or TC_INT32; signed,
 * two's complement and not DC-shifted, with bits | TC_SIGNED) -> DC
 * shift and forward colour transform -> TC_INT32 (RCT/DC) or TC_FLOAT32
 * (ICT, or DC to float) planes.  Replaces the rct_kernel, ict_kernel and
 * fdc_level_shift_kernel kernels (preprocess_rct.cl, preprocess_ict.cl,
 * preprocess_dc_level_shift.cl) and Preprocessor::dc_level_shifting. */
int tc_color_forward(tc_ctx *ctx, int kind, int ncomp,
                     const void *const *d_in, int in_type, int in_pitch,
                     void *const *d_out, int out_type, int out_pitch,
                     int w, int h, int bits);

/* ---- codestream parsing (the Tier-2 hand-off) ---------------------------- */

/* Image information from the main header.  Components share depth,
 * decomposition levels and wavelet; their code-block sizes and steps may
 * differ (COC / QCC, main or tile-part header), and cblk_w/cblk_h,
 * guard_bits and quant_style report the COD / QCD values.  Components may
 * be subsampled (single-tile images at the origin): planar outputs then
 * hold each component at its own size, one after the other. */
typedef struct tc_image_info {
    int32_t width, height, ncomp, bits;    /* width/height: Xsiz-XOsiz, Ysiz-YOsiz */
    int32_t is_signed;
    int32_t levels;                        /* decomposition levels NL */
    int32_t reversible;                    /* 1 = 5/3, 0 = 9/7 */
    int32_t mct;                           /* multiple component transform */
    int32_t cblk_w, cblk_h;
    int32_t layers, progression;
    int32_t guard_bits, quant_style;
    uint32_t ncblk;                        /* code-blocks over all components */
    uint32_t ntiles;                       /* tiles (ISO B.3); 1 for an untiled image */
    uint8_t  comp_dx[4], comp_dy[4];       /* component subsampling XRsiz / YRsiz:
                                              component c is a ceil(width/dx) x
                                              ceil(height/dy) plane */
} tc_image_info;

/* One tile of a parsed image: its region in samples from the image's
 * top-left corner, and the element offset of its coefficients in the
 * image's coefficient arena.  The arena is tile-major: tile t's component c
 * is a w*h plane (pitch w) at coef_off + c*w*h.  Tiles follow the reference's
 * type_tile geometry (codestream_image.c:256-270, tlx/tly/width/height) with
 * the SIZ offsets of ISO B.3.  Tiled images are decoded when every tile's
 * origin on the reference grid is a multiple of 2^levels in both axes (all
 * power-of-two tile sizes of at least 2^levels); others are
 * TC_E_UNSUPPORTED. */
typedef struct tc_tile_info {
    int32_t x0, y0, w, h;
    uint64_t coef_off;
} tc_tile_info;

/* Read the main header only (tile grid included).  Replaces read_main_header
 * (codestream.c:233-258). */
int tc_j2k_read_header(const uint8_t *h_cs, size_t len, tc_image_info *info);

/* Parse a whole codestream into code-block descriptors.  Segment offsets
 * refer to h_pool: for single-layer streams h_pool is the codestream itself
 * (zero copy) and *pool_is_cs is set; otherwise the parser gathers each
 * block's layers into a contiguous pool it owns.  Output offsets address the
 * image's tile-major coefficient arena (see tc_tile_info; an untiled image is
 * one tile, so plane c starts at element c*width*height).  Descriptors come
 * tile by tile.  Replaces decode_codestream / decode_tiles /
 * decode_packet_header / decode_packet_body (codestream.c:336-536) and the
 * codeBlockCallback hand-off.  Free with tc_j2k_parsed_free. */
typedef struct tc_j2k_parsed {
    tc_image_info info;
    tc_cblk_desc *desc;      /* info.ncblk entries */
    const uint8_t *pool;     /* segment pool (host) */
    uint64_t pool_len;
    int32_t pool_is_cs;
    int32_t reserved;
    const tc_tile_info *tiles;  /* info.ntiles entries, raster order */
} tc_j2k_parsed;
int tc_j2k_parse(const uint8_t *h_cs, size_t len, tc_j2k_parsed **out);
void tc_j2k_parsed_free(tc_j2k_parsed *p);

/* ---- whole-image decode (Decoder) ---------------------------------------- */

/* Decode a codestream held in host memory into host memory: planar
 * components, TC_U8 samples when bits <= 8 else TC_U16, component c at
 * h_out + c*width*height*bytes.  Runs Tier-1 with fused dequantisation, the
 * reverse DWT and the fused inverse colour transform / DC shift on the GPU.
 * Replaces Decoder::decode (Decoder.cpp:94-217).  Every entry point that
 * takes a codestream (here, tc_decode_j2k_file, tc_j2k_parse,
 * tc_j2k_read_header, tc_plan_create/rebuild) also takes a JP2 file and
 * decodes its first codestream box, as Decoder::decode does for .jp2 files
 * through jp2_parse_boxes (boxes.c:265-307). */
int tc_decode_j2k(tc_ctx *ctx, const uint8_t *h_cs, size_t len,
                  void *h_out, size_t out_bytes, tc_image_info *info);

/* Same, reading the codestream from a file (Decoder::decode(fileName)). */
int tc_decode_j2k_file(tc_ctx *ctx, const char *path, void *h_out,
                       size_t out_bytes, tc_image_info *info);

/* Device-resident plans: parse and upload once, execute many times.  A batch
 * plan merges the code-blocks of all images into one Tier-1 launch and the
 * DWT levels of all images into one launch per level. */
typedef struct tc_plan tc_plan;
int tc_plan_create(tc_ctx *ctx, const uint8_t *const *h_cs, const size_t *lens,
                   int nimages, tc_plan **out);
int tc_plan_destroy(tc_plan *plan);
/* Re-parse a plan for new codestreams, reusing its device buffers (they only
 * grow): a serving loop keeps its coefficient, scratch and pool buffers
 * resident across batches.  Waits for the plan's previous execute. */
int tc_plan_rebuild(tc_plan *plan, const uint8_t *const *h_cs, const size_t *lens,
                    int nimages);
/* tc_plan_rebuild from codestreams parsed beforehand with tc_j2k_parse (on
 * any host thread, e.g. as requests arrive), so that the rebuild itself only
 * lays out and uploads.  The parsed objects (and, for single-layer streams,
 * the codestream bytes they point into) must stay alive until the rebuild
 * returns.  No counterpart in the reference, whose parser runs inline in
 * Decoder::decode (Decoder.cpp:94-217). */
int tc_plan_rebuild_parsed(tc_plan *plan, const tc_j2k_parsed *const *parsed, int nimages);
/* Bytes of output for image i (planar, sample type as tc_decode_j2k). */
int tc_plan_output_bytes(const tc_plan *plan, int image, size_t *bytes);
int tc_plan_image_info(const tc_plan *plan, int image, tc_image_info *info);
/* Run the decode of every image in the plan; image i goes to d_out[i]
 * (device memory of tc_plan_output_bytes bytes).  Stream-ordered. */
int tc_plan_execute(tc_plan *plan, void *const *d_out);
/* Replay execute as CUDA graphs (on = 1), one per shape bucket.  In graph
 * mode the kernels read everything that changes with the images and the
 * outputs from plan buffers (descriptors, order, segment pool, and a DWT job
 * table holding the output pointers, uploaded before the launch), so a graph
 * is keyed by the launch shape: buffer addresses, Tier-1 class sizes and the
 * list of DWT launches.  The first execute of a new bucket runs normally and
 * captures the same work (Tier-1 class launches with their fork/join,
 * counter resets and every DWT level); an execute with the same key, new
 * outputs included, launches the graph; a batch rebuilt with the same launch
 * topology (the same Tier-1 classes and DWT launch kinds) updates a cached
 * graph's parameters (cudaGraphExecUpdate) instead of instantiating one.  Up
 * to 8 graphs are kept per plan, least recently used dropped; profiling
 * bypasses them, on = 0 drops them.  No counterpart in the reference. */
int tc_plan_set_graph(tc_plan *plan, int on);
/* Graph-mode counters of a plan: graphs captured and instantiated, graphs
 * updated in place for a batch of the same topology, and replays of a
 * cached graph. */
int tc_plan_graph_stats(const tc_plan *plan, uint64_t *captures, uint64_t *updates, uint64_t *replays);
/* Device memory the plan holds now (segment pool, descriptors, order,
 * coefficient arena, DWT scratch, job table; the buffers only grow).  A
 * serving loop checks its admission estimates against it.  No counterpart
 * in the reference, which allocates per call. */
int tc_plan_device_bytes(const tc_plan *plan, size_t *bytes);
/* Record CUDA events around the stages of every execute (on = 1): the
 * Tier-1 launch and the DWT/colour launches.  tc_plan_stage_ms waits for the
 * last execute and returns the device time of each stage in milliseconds.
 * (The reference times only the enqueue, CoefficientCoder.cpp:239-250,
 * defect D19.) */
int tc_plan_set_profiling(tc_plan *plan, int on);
int tc_plan_stage_ms(tc_plan *plan, float *t1_ms, float *dwt_ms);

/* ---- harness encoder (test and benchmark input generation) --------------- */

typedef struct tc_encode_params {
    int32_t width, height, ncomp, bits;
    int32_t levels;        /* decomposition levels */
    int32_t reversible;    /* 1 = 5/3 lossless, 0 = 9/7 */
    int32_t mct;           /* RCT/ICT on components 0-2 */
    int32_t cblk_log2;     /* code-block size 2^cblk_log2 (2..6) */
    double  base_step;     /* irreversible: step relative to 2^bits, divided
                              by the subband's synthesis L2 norm */
    int32_t guard_bits;    /* 0 = choose automatically */
    int32_t progression;   /* 0 LRCP, 1 RLCP, 2 RPCL, 3 PCRL, 4 CPRL */
    int32_t threads;       /* <= 0: all cores */
    int32_t is_signed;     /* signed samples (TC_S8 / TC_S16 style two's
                              complement input, no DC level shift) */
    /* Per-component overrides (0: the values above), written as COC and QCC
     * marker segments: the code-block size exponent and a multiplier of the
     * irreversible step. */
    int32_t comp_cblk_log2[4];
    double  comp_step_scale[4];
    /* Component subsampling XRsiz / YRsiz (0: 1).  Component c is a
     * ceil(width/dx) x ceil(height/dy) plane; the planes follow one another.
     * The colour transform needs components 0-2 at one size. */
    int32_t comp_dx[4], comp_dy[4];
    /* Code-block style bits (TC_CBLK_STYLE_*) for COD's SPcod; PTERM is
     * accepted and written, the terminations are the plain ones (ISO D.4.2
     * allows either encoder). The GPU encoder takes 0 only. */
    int32_t cblk_style;
    /* Quality layers (0 or 1: one).  Each block's passes are split evenly
     * over the layers; a codeword segment that a layer boundary cuts is
     * split by bytes in proportion, so every layer together gives the whole
     * codeword (no rate-distortion truncation points). */
    int32_t layers;
    /* Packet headers: 0 in the packets, 1 packed into PPT marker segments of
     * the tile-part header, 2 packed into PPM marker segments of the main
     * header (ISO A.7.4-A.7.5). */
    int32_t packed_headers;
    /* Region of interest [roi_x0, roi_x1) x [roi_y0, roi_y1) in image
     * samples (empty: none), coded with the maxshift method (RGN, ISO
     * Annex H): per component, the shift is the bit count of the largest
     * background magnitude. */
    int32_t roi_x0, roi_y0, roi_x1, roi_y1;
} tc_encode_params;

/* Encode planar samples (8-bit when bits <= 8, else 16-bit; unsigned, or
 * two's complement when is_signed) into a single-tile codestream with all
 * coding passes in p.layers quality layers (a harness encoder: the
 * reference has none). */
int tc_encode_j2k(const tc_encode_params *p, const void *h_planes,
                  uint8_t *h_out, size_t cap, size_t *out_len);

/* ---- GPU Tier-1 encoder (no counterpart in the reference, which decodes
 *      only) -------------------------------------------------------------- */

/* One code-block to encode: its samples in the input plane set, its band. */
typedef struct tc_t1_enc_desc {
    uint64_t in_off;     /* element offset of sample (0,0) */
    uint32_t in_pitch;   /* row pitch in elements */
    float    inv_step;   /* TC_CBLK_IRREVERSIBLE: 1 / step of the band */
    uint16_t w, h;       /* 1..64 */
    uint8_t  orient;     /* 0 LL, 1 HL, 2 LH, 3 HH */
    uint8_t  mb;         /* magnitude bit-planes Mb of the band (1..31) */
    uint8_t  flags;      /* TC_CBLK_IRREVERSIBLE: float input, quantised
                            floor(|x| / step); else int32 quantised input */
    uint8_t  max_passes; /* coding passes to keep, the codeword terminated
                            after the last (0 or more than the block has:
                            all of them) */
} tc_t1_enc_desc;

typedef struct tc_t1_enc_result {
    uint32_t len;            /* codeword bytes */
    uint32_t passes;         /* coding passes kept */
    uint32_t zero_bitplanes; /* Mb - coded bit-planes */
    uint32_t status;         /* 0 ok, 1 bad descriptor, 2 magnitude above
                                2^Mb, 3 codeword longer than cap */
} tc_t1_enc_result;

/* The whole encoder on the GPU: the forward colour transform with the DC
 * shift, the forward DWT levels, deadzone quantisation and Tier-1 per
 * code-block run as kernels; the host assembles packets and headers from
 * the codewords (as tc_encode_j2k does).  Lossless output is byte-identical
 * to tc_encode_j2k's; lossy output differs only where the fp32 DWT of the
 * GPU and the fp64 one of the host quantise a coefficient differently.
 * Same parameters and output as tc_encode_j2k. */
int tc_encode_j2k_gpu(tc_ctx *ctx, const tc_encode_params *p, const void *h_planes,
                      uint8_t *h_out, size_t cap, size_t *out_len);

/* Encode n code-blocks on the GPU, one warp each: block i's codeword (its
 * first max_passes coding passes, or all, MQ FLUSH termination) goes to
 * d_out + i*cap, its result to d_res[i].  Bit-exact with
 * tc_t1_encode_block on the same quantised coefficients and pass count.
 * Stream-ordered. */
int tc_t1_encode(tc_ctx *ctx, const tc_t1_enc_desc *d_desc, int n, const void *d_in,
                 uint8_t *d_out, uint32_t cap, tc_t1_enc_result *d_res);

/* Encode one code-block of quantised coefficients (row-major int32, w x h)
 * with the MQ coder, keeping the first `passes` coding passes (0 or more
 * than available = all) and terminating the codeword there.  Returns the
 * codeword length in *len, the pass count in *passes_out and the leading
 * zero bit-planes relative to mb in *zero_bitplanes. */
int tc_t1_encode_block(const int32_t *h_coef, int w, int h, int orient, int mb,
                       int passes, uint8_t *h_out, int cap, int *len,
                       int *passes_out, int *zero_bitplanes);

#ifdef __cplusplus
}
#endif
#endif /* TC_J2K_H */
