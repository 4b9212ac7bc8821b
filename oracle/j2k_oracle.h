/*
 * j2k_oracle.h -- CPU oracle for the JPEG 2000 decode hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain-C restatement of the
 * ISO/IEC 15444-1 algorithms that kgmoore/ThousandthChicken implements in its
 * OpenCL kernels.  It exists so that tests, the smoke check and the CPU
 * baseline leg of the benchmark can check the CUDA product path.  Nothing in
 * the product (the thousandthchicken_b200 package and libtc_j2k.so) links,
 * imports or calls it.
 *
 * Every function names the reference code it restates (paths are relative to
 * the reference project's ThousandthChicken/ directory).
 *
 * Conventions
 *   - Code-block coefficients are row-major, w*h, with w,h <= 64.
 *   - orient: 0 = LL, 1 = HL, 2 = LH, 3 = HH (codestream_image_types.h:24-27).
 *   - numbps = number of coded magnitude bit-planes = Mb - zero_bitplanes
 *     (codestream.c:411-421).
 */
#ifndef TC_J2K_ORACLE_H
#define TC_J2K_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Tier-1 (ISO Annex C MQ decoder + Annex D EBCOT passes) ------------- */

/* Decode one code-block segment.
 *   seg/len      : MQ codeword (code-block style 0: one codeword, no bypass)
 *   w,h          : block size (1..64)
 *   orient       : subband orientation (0 LL, 1 HL, 2 LH, 3 HH)
 *   numbps       : coded bit-planes (0..31)
 *   passes       : coding passes to decode (0..3*numbps-2)
 * Outputs (w*h each, row-major, pitch w):
 *   q            : signed value: sign * magnitude, magnitude bits at their
 *                  true bit-plane positions, undecoded bits zero
 *   undecoded    : per coefficient the number of low bit-planes that were not
 *                  decoded (0 when every pass was decoded); may be NULL
 * Returns 0, or a negative value for invalid arguments.
 * Restates coefficient_coder.cl:105-252 (MQ) and :471-819 (passes), with the
 * pass count honoured and state bits actually written (defects D1-D3 fixed). */
int or_t1_decode(const uint8_t *seg, int len, int w, int h, int orient,
                 int numbps, int passes, int32_t *q, uint8_t *undecoded);

/* Code-block style bits (SPcod, ISO Table A.19). */
#define OR_STYLE_BYPASS  0x01
#define OR_STYLE_RESET   0x02
#define OR_STYLE_TERMALL 0x04
#define OR_STYLE_VSC     0x08
#define OR_STYLE_PTERM   0x10
#define OR_STYLE_SEGSYM  0x20

/* Whether coding pass t (0: the first cleanup pass) ends a codeword segment
 * (ISO D.4.2, D.6), and how many segments passes [0, passes) span. */
int or_pass_terminates(int style, int t);
int or_pass_segments(int style, int passes);

/* or_t1_decode under code-block style `style`: with BYPASS or TERMALL the
 * codeword is nseg terminated segments of lens[k] bytes one after the other
 * (nseg = or_pass_segments(style, passes)), else lens is NULL.  Returns -3
 * for segment lengths that run past len. */
int or_t1_decode_style(const uint8_t *seg, int len, int w, int h, int orient,
                       int numbps, int passes, int style, const uint32_t *lens,
                       int nseg, int32_t *q, uint8_t *undecoded);

/* Same decode, written in the reference kernel's output format: 32-bit
 * sign-magnitude with the sign at bit 31 and magnitude bit b of the
 * coefficient at bit b + 31 - mb (coefficient_coder.cl:605-626,805-816).
 * out has pitch out_pitch (elements). */
int or_t1_decode_raw(const uint8_t *seg, int len, int w, int h, int orient,
                     int mb, int zero_bitplanes, int passes,
                     uint32_t *out, int out_pitch);

/* ---- Dequantisation (ISO E.1; Quantizer.cpp:37-65) ----------------------- */

/* Reversible: out = sign * (|q| + floor(r * 2^u)) for q != 0. */
void or_dequant_int(const int32_t *q, const uint8_t *undecoded, int n,
                    float r, int32_t *out);
/* Irreversible: out = sign * (|q| + r * 2^u) * step for q != 0 (double
 * arithmetic, rounded once to float). */
void or_dequant_float(const int32_t *q, const uint8_t *undecoded, int n,
                      float r, double step, float *out);
/* Reference lossless kernel semantics on sign-magnitude words
 * (quantizer_lossless_inverse.cl:31, defect D4 fixed): value = sign * (mag >> (31-mb)). */
void or_dequant_raw_int(const uint32_t *raw, int n, int mb, int32_t *out);

/* ---- DWT (ISO Annex F; dwt_transform_buffer.cl:102-489, dwt_io.cl:7-38) --- */

/* Rounding of the 5/3 lifting steps: 0 = ISO floor (>>), 1 = C truncating
 * division as in the reference kernels (defect D13). */
enum { OR_ROUND_FLOOR = 0, OR_ROUND_TRUNC = 1 };

/* Multi-level 2-D transforms on a w x h plane in Mallat layout (pitch =
 * elements per row).  Forward: vertical then horizontal per level (ISO F.4,
 * 2D_SD).  Reverse: horizontal then vertical per level (ISO F.3, 2D_SR).
 * Whole-sample symmetric extension with full periodic reflection (ISO F.3.7),
 * signals start at index 0 (tile origin at 0). */
void or_fdwt53(int32_t *x, int w, int h, int pitch, int levels, int rounding);
void or_idwt53(int32_t *x, int w, int h, int pitch, int levels, int rounding);
void or_fdwt97(double *x, int w, int h, int pitch, int levels);
void or_idwt97(double *x, int w, int h, int pitch, int levels);

/* Synthesis basis-function L2 norm of a subband of the 9/7 (wavelet=1) or 5/3
 * (wavelet=0) transform: level >= 1, orient 1..3; orient 0 = LL at that level. */
double or_subband_norm(int wavelet, int level, int orient);

/* ---- Colour + DC level shift (ISO G.1-G.2; preprocess_*.cl) -------------- */

/* Forward: samples (unsigned, bit depth bits) -> DC shifted, RCT.  In place on
 * three int32 planes of n samples (preprocess_rct.cl:18-31). */
void or_rct_forward(int32_t *c0, int32_t *c1, int32_t *c2, size_t n, int bits);
/* Inverse RCT + DC shift + clamp to [0, 2^bits-1] (preprocess_rct_inverse.cl:18-36). */
void or_rct_inverse(int32_t *c0, int32_t *c1, int32_t *c2, size_t n, int bits);
/* Forward ICT in double after DC shift (preprocess_ict.cl:20-37, without the
 * rounding to int). */
void or_ict_forward(const int32_t *r, const int32_t *g, const int32_t *b,
                    double *y, double *cb, double *cr, size_t n, int bits);
/* Inverse ICT (ISO G.2 coefficients, not the reference's defective constants,
 * defect D9) + round half to even + DC shift + clamp. */
void or_ict_inverse(const double *y, const double *cb, const double *cr,
                    int32_t *r, int32_t *g, int32_t *b, size_t n, int bits);
/* DC shift only (preprocess_dc_level_shift*.cl). */
void or_dc_forward(int32_t *x, size_t n, int bits);
void or_dc_inverse_clamp(int32_t *x, size_t n, int bits);
/* Float sample -> round half to even, DC shift, clamp. */
void or_dc_inverse_float(const double *x, int32_t *out, size_t n, int bits);

/* ---- Whole-tile decode from code-block descriptors ----------------------- */

/* A code-block as produced by Tier-2 parsing (the descriptor the product's
 * C ABI also takes; field meaning documented in include/tc_j2k.h). */
typedef struct or_cblk {
    uint64_t seg_off;
    uint32_t seg_len;
    uint16_t w, h;
    uint8_t passes, mb, zero_bitplanes, orient;
    uint8_t comp, flags, style, roi;   /* style: OR_STYLE_*; roi: ROI maxshift (0: none) */
    uint32_t out_x, out_y;   /* position in the component's Mallat plane */
    float step;              /* dequantisation step (irreversible only) */
} or_cblk;

/* Decode the code-blocks into per-component Mallat planes (int32 for
 * reversible, float for irreversible), run the reverse DWT, the inverse
 * colour transform (mct: 0 none, 1 RCT/ICT by wavelet) and DC shift, and write
 * clamped samples as uint16 planes (out + c*w*h).  threads <= 0 uses all
 * cores.  Returns 0 or a negative error. */
/* Flag or-ed into `bits`: signed samples (no DC level shift, clamped to the
 * signed range; or_decode_tile's 16-bit output then holds two's complement). */
#define OR_SIGNED 0x100

int or_decode_tile(const or_cblk *cb, int n, const uint8_t *pool,
                   int w, int h, int ncomp, int bits, int levels,
                   int reversible, int mct, float r, int threads,
                   uint16_t *out);

/* ---- Encoding (the oracle's own inputs) ---------------------------------- */

/* Encode one code-block of quantised coefficients (row-major, w x h) with
 * the MQ coder of ISO C.2 and the passes of ISO D.3, keeping the first
 * `passes` coding passes (<= 0 or more than available: all of them) and
 * terminating the codeword there (FLUSH, ISO C.2.9).  Returns the codeword
 * length in *len, the passes kept and the coded bit-planes.  0, or -1 for
 * bad arguments, -2 out of memory, -3 a codeword longer than cap.  The
 * reference decodes only; this is the standard's encoder. */
int or_t1_encode(const int32_t *coef, int w, int h, int orient, int passes,
                 uint8_t *out, int cap, int *len, int *passes_out, int *numbps_out);

/* Encode a w x h tile at the origin from planar unsigned samples
 * (ncomp * w * h): DC shift, forward RCT (reversible) or ICT (irreversible)
 * on components 0-2 when mct, `levels` of forward 5/3 or 9/7 (FP64),
 * deadzone quantisation with the step of each band derived from base_step *
 * 2^bits / (its 9/7 synthesis L2 norm) and rounded to its ISO E.1 (exponent,
 * mantissa) code, and cblk x cblk code-blocks with every pass kept.  Returns
 * malloc'd code-block descriptors (mb = 31) and a 16-byte aligned segment
 * pool; free both with or_encoded_free.  0, or a negative error. */
int or_encode_tile(const uint16_t *samples, int w, int h, int ncomp, int bits,
                   int levels, int reversible, int mct, double base_step, int cblk,
                   int threads, or_cblk **cb_out, int *n_out, uint8_t **pool_out,
                   size_t *pool_len_out);
void or_encoded_free(or_cblk *cb, uint8_t *pool);

/* or_decode_tile, also returning (when out_f64 is not NULL and the tile is
 * irreversible) the FP64 samples after the inverse colour transform and the
 * DC shift, before rounding and clamping (ncomp * w * h doubles). */
int or_decode_tile_f64(const or_cblk *cb, int n, const uint8_t *pool,
                       int w, int h, int ncomp, int bits, int levels,
                       int reversible, int mct, float r, int threads,
                       uint16_t *out, double *out_f64);

/* The coefficients a decoder reconstructs from the first `passes` coding
 * passes of a block (row-major w x h, pitch w): derived from the
 * coefficients and the pass membership rules of ISO D.3 alone, with no MQ
 * coding, as the independent statement of "the truncated coefficients".
 * passes <= 0 gives zeros; all passes give the coefficients. */
void or_t1_truncate(const int32_t *coef, int w, int h, int passes, int32_t *out);
/* The same over n blocks, block i at element offset off[i] (pitch w[i]) of
 * coef and of out, on `threads` threads (<= 0: all cores). */
void or_t1_truncate_batch(const int32_t *coef, const uint64_t *off, const uint16_t *w, const uint16_t *h,
                          const uint8_t *passes, int n, int threads, int32_t *out);

#ifdef __cplusplus
}
#endif
#endif
