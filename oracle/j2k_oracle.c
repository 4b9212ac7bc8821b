/*
 * j2k_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY) for the JPEG 2000
 * decode hot path: a direct, unoptimised restatement of ISO/IEC 15444-1
 * Annexes C (MQ coder), D (EBCOT Tier-1), E (quantisation), F (DWT) and
 * G (colour transforms), following the stages of kgmoore/ThousandthChicken.
 * Only tests, the smoke check and the benchmark's CPU-baseline leg use it.
 *
 * Reference files restated (paths relative to ThousandthChicken/):
 *   coefficient_coder.cl:36-60    MQ probability tables (Qe/NMPS/NLPS/SWITCH)
 *   coefficient_coder.cl:105-252  bytein/renormd/lps_exchange/mps_exchange/
 *                                 mqInitDec/mqDecode
 *   coefficient_coder.cl:271-469  context formation (ZC/SC/MR labels)
 *   coefficient_coder.cl:471-819  RL/significance/sign functors, the three
 *                                 passes and g_decode's bit-plane loop
 *   quantizer_*_inverse.cl, Quantizer.cpp:37-65   dequantisation
 *   dwt_transform_buffer.cl:102-489, dwt_io.cl:7-38  lifting and mirroring
 *   preprocess_*.cl               colour transforms and DC level shift
 * The code-block style modes (ISO D.4-D.6: bypass, context reset,
 * termination on every pass, vertically causal contexts, segmentation
 * symbols) have no counterpart in the reference, which decodes style 0 only;
 * they follow the standard and are pinned against OpenJPEG's decoder.
 */
#include "j2k_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* Minimal parallel-for over [0, n) on POSIX threads (items claimed with an
 * atomic counter).  threads <= 0 uses every online core. */
typedef struct {
    void (*fn)(void *arg, int i);
    void *arg;
    int n;
    int next;
} or_pool;

static void *or_worker(void *p)
{
    or_pool *pl = (or_pool *)p;
    for (;;) {
        const int i = __atomic_fetch_add(&pl->next, 1, __ATOMIC_RELAXED);
        if (i >= pl->n) break;
        pl->fn(pl->arg, i);
    }
    return NULL;
}

static void or_parallel_for(int n, int threads, void (*fn)(void *, int), void *arg)
{
    or_pool pl = {fn, arg, n, 0};
    pthread_t tid[256];
    int nt = threads > 0 ? threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nt < 1) nt = 1;
    if (nt > 256) nt = 256;
    if (nt > n) nt = n;
    if (nt <= 1) {
        or_worker(&pl);
        return;
    }
    for (int t = 0; t < nt; t++)
        if (pthread_create(&tid[t], NULL, or_worker, &pl)) { nt = t; break; }
    for (int t = 0; t < nt; t++) pthread_join(tid[t], NULL);
    if (nt == 0) or_worker(&pl);
}

/* ===================== MQ decoder (ISO C.3) ============================== */

/* ISO Table C.2, the same values as coefficient_coder.cl:36-60. */
static const uint16_t kQe[47] = {
    0x5601, 0x3401, 0x1801, 0x0AC1, 0x0521, 0x0221, 0x5601, 0x5401, 0x4801, 0x3801,
    0x3001, 0x2401, 0x1C01, 0x1601, 0x5601, 0x5401, 0x5101, 0x4801, 0x3801, 0x3401,
    0x3001, 0x2801, 0x2401, 0x2201, 0x1C01, 0x1801, 0x1601, 0x1401, 0x1201, 0x1101,
    0x0AC1, 0x09C1, 0x08A1, 0x0521, 0x0441, 0x02A1, 0x0221, 0x0141, 0x0111, 0x0085,
    0x0049, 0x0025, 0x0015, 0x0009, 0x0005, 0x0001, 0x5601};
static const uint8_t kNMPS[47] = {
    1, 2, 3, 4, 5, 38, 7, 8, 9, 10, 11, 12, 13, 29, 15, 16, 17, 18, 19, 20,
    21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39, 40,
    41, 42, 43, 44, 45, 45, 46};
static const uint8_t kNLPS[47] = {
    1, 6, 9, 12, 29, 33, 6, 14, 14, 14, 17, 18, 20, 21, 14, 14, 15, 16, 17, 18,
    19, 19, 20, 21, 22, 23, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37,
    38, 39, 40, 41, 42, 43, 46};
static const uint8_t kSWITCH[47] = {
    1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0,
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
    0, 0, 0, 0, 0, 0, 0};

/* Context labels (ISO D.3): 0-8 zero coding, 9-13 sign coding, 14-16
 * magnitude refinement, 17 uniform, 18 run-length
 * (coefficient_coder.cl:64-65 names CX_UNI 17 and CX_RUN 18). */
enum { CX_UNI = 17, CX_RUN = 18, NCX = 19 };

typedef struct {
    const uint8_t *d;
    int len, bp, ct;
    uint32_t a, c;
    uint8_t idx[NCX], mps[NCX];
    /* raw (bypass) segment: the bits of d MSB first (ISO D.6) */
    int raw, rct;
    uint32_t rbyte;
} mqdec;

static inline uint32_t mq_byte(const mqdec *m, int i)
{
    /* Bytes past the segment read as 0xFF: the decoder then sees a marker and
     * feeds 1-bits (ISO C.3.4; coefficient_coder.cl:124-125). */
    return (i < m->len) ? m->d[i] : 0xFFu;
}

static void mq_bytein(mqdec *m)
{
    if (mq_byte(m, m->bp) == 0xFF) {
        if (mq_byte(m, m->bp + 1) > 0x8F) {
            m->c += 0xFF00;
            m->ct = 8;
        } else {
            m->bp++;
            m->c += mq_byte(m, m->bp) << 9;
            m->ct = 7;
        }
    } else {
        m->bp++;
        m->c += mq_byte(m, m->bp) << 8;
        m->ct = 8;
    }
}

/* The decoder's registers at the start of a codeword segment (INITDEC, ISO
 * C.3.5); the contexts are left as they are. */
static void mq_start(mqdec *m, const uint8_t *d, int len)
{
    m->d = d;
    m->len = len;
    m->bp = 0;
    m->raw = 0;
    m->c = mq_byte(m, 0) << 16;
    mq_bytein(m);
    m->c <<= 7;
    m->ct -= 7;
    m->a = 0x8000;
}

/* A raw segment: bits MSB first; a byte after 0xFF holds 7 bits (its MSB is
 * a stuffed 0), and after 0xFF a byte above 0x8F is a marker that is not
 * consumed: 1-bits are read from there on, as past the end. */
static void raw_start(mqdec *m, const uint8_t *d, int len)
{
    m->d = d;
    m->len = len;
    m->bp = 0;
    m->raw = 1;
    m->rct = 0;
    m->rbyte = 0;
}

static int raw_bit(mqdec *m)
{
    if (m->rct == 0) {
        const uint32_t b = mq_byte(m, m->bp);
        if (m->rbyte == 0xFF && b > 0x8F) {
            m->rct = 8;  /* rbyte stays 0xFF */
        } else {
            m->rct = m->rbyte == 0xFF ? 7 : 8;
            m->rbyte = b;
            m->bp++;
        }
    }
    m->rct--;
    return (int)((m->rbyte >> m->rct) & 1u);
}

/* Initial context states: ISO Table D.7; mqResetDec, coefficient_coder.cl:158-172. */
static void mq_reset(mqdec *m)
{
    memset(m->idx, 0, sizeof m->idx);
    memset(m->mps, 0, sizeof m->mps);
    m->idx[0] = 4;
    m->idx[CX_RUN] = 3;
    m->idx[CX_UNI] = 46;
}

static void mq_renorm(mqdec *m)
{
    do {
        if (m->ct == 0) mq_bytein(m);
        m->a <<= 1;
        m->c <<= 1;
        m->ct--;
    } while ((m->a & 0x8000) == 0);
}

static int mq_decode(mqdec *m, int cx)
{
    const int s = m->idx[cx];
    const uint32_t qe = kQe[s];
    int d;
    m->a -= qe;
    if ((m->c >> 16) < qe) {
        /* LPS_EXCHANGE */
        if (m->a < qe) {
            d = m->mps[cx];
            m->idx[cx] = kNMPS[s];
        } else {
            d = 1 - m->mps[cx];
            if (kSWITCH[s]) m->mps[cx] ^= 1;
            m->idx[cx] = kNLPS[s];
        }
        m->a = qe;
        mq_renorm(m);
    } else {
        m->c -= qe << 16;
        if ((m->a & 0x8000) == 0) {
            /* MPS_EXCHANGE */
            if (m->a < qe) {
                d = 1 - m->mps[cx];
                if (kSWITCH[s]) m->mps[cx] ^= 1;
                m->idx[cx] = kNLPS[s];
            } else {
                d = m->mps[cx];
                m->idx[cx] = kNMPS[s];
            }
            mq_renorm(m);
        } else {
            d = m->mps[cx];
        }
    }
    return d;
}

/* One decision of a pass: raw in a bypass segment, else MQ with context cx. */
static int dec_bit(mqdec *m, int cx)
{
    return m->raw ? raw_bit(m) : mq_decode(m, cx);
}

/* ===================== Tier-1 decoder (ISO D) ============================ */

/* Zero-coding context from neighbour significance counts, ISO Table D.1
 * (the reference encodes the same table as SPCXLUT, coefficient_coder.cl:330-393). */
static int zc_context(int orient, int h, int v, int d)
{
    if (orient == 1) { int t = h; h = v; v = t; } /* HL: swap roles */
    if (orient == 3) {
        const int hv = h + v;
        if (d >= 3) return 8;
        if (d == 2) return hv >= 1 ? 7 : 6;
        if (d == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
        return hv >= 2 ? 2 : (hv == 1 ? 1 : 0);
    }
    if (h == 2) return 8;
    if (h == 1) return v >= 1 ? 7 : (d >= 1 ? 6 : 5);
    if (v == 2) return 4;
    if (v == 1) return 3;
    return d >= 2 ? 2 : (d == 1 ? 1 : 0);
}

typedef struct {
    int w, h, W;          /* W = padded row stride (w + 2) */
    uint8_t *sig, *sgn, *ref, *vis;
    int32_t *mag;
    int vsc;              /* vertically causal contexts (ISO D.7) */
} t1st;

#define AT(st, arr, x, y) ((st)->arr[((y) + 1) * (st)->W + (x) + 1])

/* Whether row y's neighbours in row y + 1 count: not across a stripe
 * boundary under vertically causal contexts. */
static inline int below_seen(const t1st *s, int y) { return !(s->vsc && (y & 3) == 3); }

static void nb_counts(const t1st *s, int x, int y, int *h, int *v, int *d)
{
    const int b = below_seen(s, y);
    *h = AT(s, sig, x - 1, y) + AT(s, sig, x + 1, y);
    *v = AT(s, sig, x, y - 1) + (b ? AT(s, sig, x, y + 1) : 0);
    *d = AT(s, sig, x - 1, y - 1) + AT(s, sig, x + 1, y - 1) +
         (b ? AT(s, sig, x - 1, y + 1) + AT(s, sig, x + 1, y + 1) : 0);
}

/* Sign coding, ISO Tables D.2/D.3 (signcxlut, coefficient_coder.cl:406-435). */
static int decode_sign(mqdec *m, const t1st *s, int x, int y)
{
    int hc = 0, vc = 0, cx, xr;
#define CONTRIB(xx, yy) (AT(s, sig, xx, yy) ? (AT(s, sgn, xx, yy) ? -1 : 1) : 0)
    if (m->raw) return raw_bit(m); /* bypass: the sign bit itself */
    hc = CONTRIB(x - 1, y) + CONTRIB(x + 1, y);
    vc = CONTRIB(x, y - 1) + (below_seen(s, y) ? CONTRIB(x, y + 1) : 0);
#undef CONTRIB
    hc = hc > 1 ? 1 : (hc < -1 ? -1 : hc);
    vc = vc > 1 ? 1 : (vc < -1 ? -1 : vc);
    if (hc == 0) {
        cx = vc == 0 ? 9 : 10;
        xr = vc < 0;
    } else {
        /* (H,V) = (1,1)->13 (1,0)->12 (1,-1)->11, mirrored with XOR 1 for H = -1 */
        cx = 12 + hc * vc;
        xr = hc < 0;
    }
    return mq_decode(m, cx) ^ xr;
}

static void become_significant(mqdec *m, t1st *s, int x, int y, int p)
{
    AT(s, sgn, x, y) = (uint8_t)decode_sign(m, s, x, y);
    AT(s, sig, x, y) = 1;
    AT(s, mag, x, y) |= (int32_t)1 << p;
}

static void pass_spp(mqdec *m, t1st *s, int orient, int p)
{
    for (int y0 = 0; y0 < s->h; y0 += 4)
        for (int x = 0; x < s->w; x++)
            for (int y = y0; y < y0 + 4 && y < s->h; y++) {
                int hh, vv, dd;
                if (AT(s, sig, x, y)) continue;
                nb_counts(s, x, y, &hh, &vv, &dd);
                if (hh + vv + dd == 0) continue;
                AT(s, vis, x, y) = 1;
                if (dec_bit(m, zc_context(orient, hh, vv, dd)))
                    become_significant(m, s, x, y, p);
            }
}

static void pass_mrp(mqdec *m, t1st *s, int p)
{
    for (int y0 = 0; y0 < s->h; y0 += 4)
        for (int x = 0; x < s->w; x++)
            for (int y = y0; y < y0 + 4 && y < s->h; y++) {
                int hh, vv, dd, cx;
                if (!AT(s, sig, x, y) || AT(s, vis, x, y)) continue;
                nb_counts(s, x, y, &hh, &vv, &dd);
                /* ISO Table D.4; getMRCX, coefficient_coder.cl:461-469. */
                cx = AT(s, ref, x, y) ? 16 : (hh + vv + dd ? 15 : 14);
                if (dec_bit(m, cx)) AT(s, mag, x, y) |= (int32_t)1 << p;
                AT(s, ref, x, y) = 1;
            }
}

static void pass_cup(mqdec *m, t1st *s, int orient, int p)
{
    for (int y0 = 0; y0 < s->h; y0 += 4)
        for (int x = 0; x < s->w; x++) {
            int y = y0;
            if (y0 + 4 <= s->h) {
                /* Run-length mode (ISO D.3.4): four in-bounds rows, none
                 * significant or visited, all with zero-coding context 0. */
                int ok = 1;
                for (int k = 0; k < 4 && ok; k++) {
                    int hh, vv, dd;
                    if (AT(s, sig, x, y0 + k) || AT(s, vis, x, y0 + k)) { ok = 0; break; }
                    nb_counts(s, x, y0 + k, &hh, &vv, &dd);
                    if (hh + vv + dd) ok = 0;
                }
                if (ok) {
                    int r;
                    if (!mq_decode(m, CX_RUN)) continue;
                    r = mq_decode(m, CX_UNI) << 1;
                    r |= mq_decode(m, CX_UNI);
                    become_significant(m, s, x, y0 + r, p);
                    y = y0 + r + 1;
                }
            }
            for (; y < y0 + 4 && y < s->h; y++) {
                int hh, vv, dd;
                if (AT(s, sig, x, y) || AT(s, vis, x, y)) continue;
                nb_counts(s, x, y, &hh, &vv, &dd);
                if (mq_decode(m, zc_context(orient, hh, vv, dd)))
                    become_significant(m, s, x, y, p);
            }
        }
}

int or_pass_terminates(int style, int t)
{
    if (style & OR_STYLE_TERMALL) return 1;
    if (style & OR_STYLE_BYPASS) return t == 9 || (t >= 10 && t % 3 != 1);
    return 0;
}

int or_pass_segments(int style, int passes)
{
    int n = passes > 0;
    for (int t = 0; t + 1 < passes; t++) n += or_pass_terminates(style, t);
    return n;
}

/* Pass t of a bypass stream is raw-coded: SPP and MRP from the 11th pass. */
static int pass_is_raw(int style, int t) { return (style & OR_STYLE_BYPASS) && t >= 10 && t % 3 != 0; }

/* Codeword segments of one block: lens[0..nseg) when given (BYPASS /
 * TERMALL), else one segment of len bytes. */
typedef struct {
    const uint8_t *seg;
    int len, style, nseg, si;
    const uint32_t *lens;
    size_t off;
} segwalk;

/* Before pass t: start the next codeword segment where one begins. */
static int begin_pass(mqdec *m, segwalk *g, int t)
{
    if (!g->lens) {
        if (t == 0) mq_start(m, g->seg, g->len);
        return 0;
    }
    if (t > 0 && !or_pass_terminates(g->style, t - 1)) return 0;
    if (t > 0) g->off += g->lens[g->si++];
    if (g->si >= g->nseg || g->off + g->lens[g->si] > (size_t)g->len) return -1;
    if (pass_is_raw(g->style, t)) raw_start(m, g->seg + g->off, (int)g->lens[g->si]);
    else mq_start(m, g->seg + g->off, (int)g->lens[g->si]);
    return 0;
}

/* Shared body of the decode entry points.  Leaves the magnitude/sign state
 * in st and returns the last pass type (0 CUP, 1 SPP, 2 MRP) and the plane
 * it ran on, -1 when no pass ran, or -2 for a bad segment table. */
static int t1_run(const uint8_t *seg, int len, int w, int h, int orient,
                  int numbps, int passes, t1st *st, int *last_plane,
                  int style, const uint32_t *lens, int nseg)
{
    mqdec m;
    segwalk g = {seg, len, style, nseg, 0, lens, 0};
    int type = -1, pi = 0;
    memset(&m, 0, sizeof m);
    mq_reset(&m);
    st->vsc = (style & OR_STYLE_VSC) != 0;
    *last_plane = numbps;
    for (int p = numbps - 1; p >= 0 && pi < passes; p--) {
        if (p != numbps - 1) {
            if (begin_pass(&m, &g, pi)) return -2;
            pass_spp(&m, st, orient, p);
            if (style & OR_STYLE_RESET) mq_reset(&m);
            type = 1; *last_plane = p;
            if (++pi >= passes) break;
            if (begin_pass(&m, &g, pi)) return -2;
            pass_mrp(&m, st, p);
            if (style & OR_STYLE_RESET) mq_reset(&m);
            type = 2;
            if (++pi >= passes) break;
        }
        if (begin_pass(&m, &g, pi)) return -2;
        pass_cup(&m, st, orient, p);
        if (style & OR_STYLE_SEGSYM) /* segmentation symbol, ISO D.5 */
            for (int k = 0; k < 4; k++) mq_decode(&m, CX_UNI);
        if (style & OR_STYLE_RESET) mq_reset(&m);
        type = 0; *last_plane = p;
        ++pi;
        memset(st->vis, 0, (size_t)(st->W) * (st->h + 2));
    }
    (void)w; (void)h;
    return type;
}

static int t1_alloc(t1st *st, int w, int h)
{
    const size_t n = (size_t)(w + 2) * (h + 2);
    st->w = w; st->h = h; st->W = w + 2;
    st->sig = calloc(n, 1); st->sgn = calloc(n, 1);
    st->ref = calloc(n, 1); st->vis = calloc(n, 1);
    st->mag = calloc(n, sizeof(int32_t));
    return (st->sig && st->sgn && st->ref && st->vis && st->mag) ? 0 : -1;
}

static void t1_free(t1st *st)
{
    free(st->sig); free(st->sgn); free(st->ref); free(st->vis); free(st->mag);
}

static int t1_args_ok(int len, int w, int h, int orient, int numbps, int passes)
{
    if (len < 0 || w < 1 || h < 1 || w > 64 || h > 64) return 0;
    if (orient < 0 || orient > 3 || numbps < 0 || numbps > 31) return 0;
    if (passes < 0 || (numbps > 0 && passes > 3 * numbps - 2)) return 0;
    return 1;
}

int or_t1_decode(const uint8_t *seg, int len, int w, int h, int orient,
                 int numbps, int passes, int32_t *q, uint8_t *undecoded)
{
    return or_t1_decode_style(seg, len, w, h, orient, numbps, passes, 0, NULL, 0, q, undecoded);
}

int or_t1_decode_style(const uint8_t *seg, int len, int w, int h, int orient,
                       int numbps, int passes, int style, const uint32_t *lens,
                       int nseg, int32_t *q, uint8_t *undecoded)
{
    t1st st;
    int last_plane, type;
    if (!t1_args_ok(len, w, h, orient, numbps, passes)) return -1;
    if (lens && nseg != or_pass_segments(style, passes)) return -1;
    if (t1_alloc(&st, w, h)) { t1_free(&st); return -2; }
    type = (numbps > 0 && passes > 0)
               ? t1_run(seg, len, w, h, orient, numbps, passes, &st, &last_plane, style, lens, nseg)
               : -1;
    if (type == -2) { t1_free(&st); return -3; }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const int32_t mg = AT(&st, mag, x, y);
            int u = 0;
            q[y * w + x] = AT(&st, sgn, x, y) ? -mg : mg;
            if (type >= 0) {
                u = last_plane;
                /* Truncated inside a bit-plane (ISO E.1.1.2, Nb(u,v)): after
                 * a significance-propagation pass only the coefficients it
                 * visited carry that plane; after a refinement pass the
                 * significant ones do too; the rest wait for the cleanup. */
                if (type == 1 && !AT(&st, vis, x, y)) u = last_plane + 1;
                if (type == 2 && !AT(&st, vis, x, y) && !AT(&st, sig, x, y)) u = last_plane + 1;
            }
            if (undecoded) undecoded[y * w + x] = (uint8_t)u;
        }
    t1_free(&st);
    return 0;
}

int or_t1_decode_raw(const uint8_t *seg, int len, int w, int h, int orient,
                     int mb, int zero_bitplanes, int passes,
                     uint32_t *out, int out_pitch)
{
    t1st st;
    int last_plane;
    const int numbps = mb - zero_bitplanes;
    if (mb < 1 || mb > 31 || zero_bitplanes < 0) return -1;
    if (!t1_args_ok(len, w, h, orient, numbps < 0 ? 0 : numbps, passes)) return -1;
    if (t1_alloc(&st, w, h)) { t1_free(&st); return -2; }
    if (numbps > 0 && passes > 0)
        t1_run(seg, len, w, h, orient, numbps, passes, &st, &last_plane, 0, NULL, 0);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const uint32_t mg = (uint32_t)AT(&st, mag, x, y);
            out[(size_t)y * out_pitch + x] =
                (mg << (31 - mb)) | ((uint32_t)AT(&st, sgn, x, y) << 31);
        }
    t1_free(&st);
    return 0;
}

/* ===================== Dequantisation (ISO E.1) ========================== */

void or_dequant_int(const int32_t *q, const uint8_t *undecoded, int n,
                    float r, int32_t *out)
{
    for (int i = 0; i < n; i++) {
        const int32_t v = q[i];
        int32_t a = v < 0 ? -v : v;
        if (a && undecoded && undecoded[i])
            a += (int32_t)floor((double)r * (double)(1u << undecoded[i]));
        out[i] = v < 0 ? -a : a;
    }
}

void or_dequant_float(const int32_t *q, const uint8_t *undecoded, int n,
                      float r, double step, float *out)
{
    for (int i = 0; i < n; i++) {
        const int32_t v = q[i];
        double a = v < 0 ? -(double)v : (double)v;
        if (a != 0.0) a += (double)r * (double)(1u << (undecoded ? undecoded[i] : 0));
        out[i] = (float)((v < 0 ? -a : a) * step);
    }
}

void or_dequant_raw_int(const uint32_t *raw, int n, int mb, int32_t *out)
{
    for (int i = 0; i < n; i++) {
        const int32_t a = (int32_t)((raw[i] & 0x7FFFFFFFu) >> (31 - mb));
        out[i] = (raw[i] >> 31) ? -a : a;
    }
}

/* ===================== DWT (ISO F) ======================================= */

/* Periodic symmetric extension index (ISO F.3.7 / F.4.7). */
static inline int pse(int i, int n)
{
    const int per = 2 * (n - 1);
    if (n == 1) return 0;
    i %= per;
    if (i < 0) i += per;
    return i >= n ? per - i : i;
}

static inline int32_t fdiv(int32_t a, int b, int rounding)
{
    if (rounding == OR_ROUND_TRUNC) return a / b;
    return (int32_t)floor((double)a / b);
}

/* 1-D reversible 5/3 on an interleaved signal (even = low, odd = high). */
static void idwt53_1d(int32_t *x, int n, int rnd)
{
    if (n < 2) return;
    for (int k = 0; k < n; k += 2)
        x[k] -= fdiv(x[pse(k - 1, n)] + x[pse(k + 1, n)] + 2, 4, rnd);
    for (int k = 1; k < n; k += 2)
        x[k] += fdiv(x[pse(k - 1, n)] + x[pse(k + 1, n)], 2, rnd);
}

static void fdwt53_1d(int32_t *x, int n, int rnd)
{
    if (n < 2) return;
    for (int k = 1; k < n; k += 2)
        x[k] -= fdiv(x[pse(k - 1, n)] + x[pse(k + 1, n)], 2, rnd);
    for (int k = 0; k < n; k += 2)
        x[k] += fdiv(x[pse(k - 1, n)] + x[pse(k + 1, n)] + 2, 4, rnd);
}

/* 9/7 lifting constants (ISO F.4.8.2; dwt_f97.cl:5-8, dwt_common.cl:10-11). */
static const double A97 = -1.586134342059924, B97 = -0.052980118572961,
                    G97 = 0.882911075530934, D97 = 0.443506852043971,
                    K97 = 1.230174104914001;

static void fdwt97_1d(double *x, int n)
{
    if (n < 2) return;
    for (int k = 1; k < n; k += 2) x[k] += A97 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 0; k < n; k += 2) x[k] += B97 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 1; k < n; k += 2) x[k] += G97 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 0; k < n; k += 2) x[k] += D97 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 1; k < n; k += 2) x[k] *= K97;
    for (int k = 0; k < n; k += 2) x[k] /= K97;
}

static void idwt97_1d(double *x, int n)
{
    if (n < 2) return;
    for (int k = 0; k < n; k += 2) x[k] *= K97;
    for (int k = 1; k < n; k += 2) x[k] /= K97;
    for (int k = 0; k < n; k += 2) x[k] -= D97 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 1; k < n; k += 2) x[k] -= G97 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 0; k < n; k += 2) x[k] -= B97 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 1; k < n; k += 2) x[k] -= A97 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
}

/* Generic level driver over strided lines: gather -> (de)interleave ->
 * 1-D transform -> scatter.  The lines of a pass are independent, so a
 * pass is split into chunks of lines over `threads` workers (the result
 * does not depend on the split). */
typedef struct {
    void *x;
    int w, h, pitch, fwd, rnd, vertical, elem;
} or_lvl_job;

enum { LINES_PER_CHUNK = 32 };

#define LEVEL_LINES(T, BODY)                                                   \
    do {                                                                       \
        T *x = (T *)J->x;                                                      \
        const int n = J->vertical ? J->h : J->w;                               \
        const int lines = J->vertical ? J->w : J->h;                           \
        const int nl = (n + 1) / 2, fwd = J->fwd, rnd = J->rnd;                \
        T *line = malloc(sizeof(T) * n), *tmp = malloc(sizeof(T) * n);        \
        (void)rnd;                                                             \
        for (int l = chunk * LINES_PER_CHUNK;                                  \
             l < lines && l < (chunk + 1) * LINES_PER_CHUNK; l++) {            \
            T *base = J->vertical ? x + l : x + (size_t)l * J->pitch;          \
            const size_t step = J->vertical ? (size_t)J->pitch : 1;            \
            for (int i = 0; i < n; i++) line[i] = base[i * step];              \
            if (fwd) {                                                         \
                BODY(line, n, 1);                                              \
                for (int i = 0; i < n; i++)                                    \
                    tmp[(i & 1) ? nl + i / 2 : i / 2] = line[i];               \
            } else {                                                           \
                for (int i = 0; i < n; i++)                                    \
                    tmp[i] = line[(i & 1) ? nl + i / 2 : i / 2];               \
                BODY(tmp, n, 0);                                               \
            }                                                                  \
            for (int i = 0; i < n; i++) base[i * step] = tmp[i];               \
        }                                                                      \
        free(line);                                                            \
        free(tmp);                                                             \
    } while (0)

#define F53(v, n, fwd) do { if (fwd) fdwt53_1d(v, n, rnd); else idwt53_1d(v, n, rnd); } while (0)
#define F97(v, n, fwd) do { if (fwd) fdwt97_1d(v, n); else idwt97_1d(v, n); } while (0)

static void or_lvl_chunk(void *arg, int chunk)
{
    const or_lvl_job *J = (const or_lvl_job *)arg;
    if (J->elem == 4) LEVEL_LINES(int32_t, F53);
    else LEVEL_LINES(double, F97);
}

/* One level: forward = columns then rows (ISO F.4, 2D_SD); reverse = rows
 * then columns (ISO F.3, 2D_SR). */
static void level_mt(void *x, int elem, int w, int h, int pitch, int fwd, int rnd, int threads)
{
    for (int pass = 0; pass < 2; pass++) {
        or_lvl_job J = {x, w, h, pitch, fwd, rnd, fwd ? (pass == 0) : (pass == 1), elem};
        const int lines = J.vertical ? w : h;
        or_parallel_for((lines + LINES_PER_CHUNK - 1) / LINES_PER_CHUNK, threads, or_lvl_chunk, &J);
    }
}

static void fdwt53_mt(int32_t *x, int w, int h, int pitch, int levels, int rounding, int threads)
{
    for (int l = 0; l < levels; l++) {
        level_mt(x, 4, w, h, pitch, 1, rounding, threads);
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
}

static void idwt53_mt(int32_t *x, int w, int h, int pitch, int levels, int rounding, int threads)
{
    int ws[33], hs[33];
    ws[0] = w; hs[0] = h;
    for (int l = 1; l <= levels; l++) { ws[l] = (ws[l - 1] + 1) / 2; hs[l] = (hs[l - 1] + 1) / 2; }
    for (int l = levels - 1; l >= 0; l--) level_mt(x, 4, ws[l], hs[l], pitch, 0, rounding, threads);
}

static void fdwt97_mt(double *x, int w, int h, int pitch, int levels, int threads)
{
    for (int l = 0; l < levels; l++) {
        level_mt(x, 8, w, h, pitch, 1, 0, threads);
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
}

static void idwt97_mt(double *x, int w, int h, int pitch, int levels, int threads)
{
    int ws[33], hs[33];
    ws[0] = w; hs[0] = h;
    for (int l = 1; l <= levels; l++) { ws[l] = (ws[l - 1] + 1) / 2; hs[l] = (hs[l - 1] + 1) / 2; }
    for (int l = levels - 1; l >= 0; l--) level_mt(x, 8, ws[l], hs[l], pitch, 0, 0, threads);
}

void or_fdwt53(int32_t *x, int w, int h, int pitch, int levels, int rounding)
{
    fdwt53_mt(x, w, h, pitch, levels, rounding, 1);
}

void or_idwt53(int32_t *x, int w, int h, int pitch, int levels, int rounding)
{
    idwt53_mt(x, w, h, pitch, levels, rounding, 1);
}

void or_fdwt97(double *x, int w, int h, int pitch, int levels)
{
    fdwt97_mt(x, w, h, pitch, levels, 1);
}

void or_idwt97(double *x, int w, int h, int pitch, int levels)
{
    idwt97_mt(x, w, h, pitch, levels, 1);
}

/* 1-D synthesis norm of a unit coefficient in the low (high = 0) or high
 * (high = 1) band at the given level, computed by running the real-valued
 * multi-level synthesis on an impulse. */
static double norm_1d(int wavelet, int level, int high)
{
    const int n = 1 << (level + 7);
    double *x = calloc((size_t)n, sizeof(double));
    double s = 0.0;
    int len = n, pos;
    for (int l = 0; l < level; l++) len = (len + 1) / 2;
    /* len = low-band length at this level; the high band of this level
     * starts right after it in the 1-D Mallat layout. */
    pos = high ? len + len / 2 : len / 2;
    x[pos] = 1.0;
    for (int l = level - 1; l >= 0; l--) {
        int m = n;
        double *t;
        for (int k = 0; k < l; k++) m = (m + 1) / 2;
        t = malloc(sizeof(double) * m);
        for (int i = 0; i < m; i++) t[i] = x[(i & 1) ? (m + 1) / 2 + i / 2 : i / 2];
        if (wavelet == 1) {
            idwt97_1d(t, m);
        } else {
            /* real-valued 5/3 synthesis (no rounding) */
            for (int k = 0; k < m; k += 2) t[k] -= 0.25 * (t[pse(k - 1, m)] + t[pse(k + 1, m)]);
            for (int k = 1; k < m; k += 2) t[k] += 0.5 * (t[pse(k - 1, m)] + t[pse(k + 1, m)]);
        }
        memcpy(x, t, sizeof(double) * m);
        free(t);
    }
    for (int i = 0; i < n; i++) s += x[i] * x[i];
    free(x);
    return sqrt(s);
}

double or_subband_norm(int wavelet, int level, int orient)
{
    const double lo = norm_1d(wavelet, level, 0), hi = norm_1d(wavelet, level, 1);
    switch (orient) {
    case 0: return lo * lo;
    case 1: return hi * lo;  /* HL: high horizontally, low vertically */
    case 2: return lo * hi;
    default: return hi * hi;
    }
}

/* ===================== Colour + DC shift (ISO G) ========================= */

static inline int32_t clampi(int32_t v, int32_t lo, int32_t hi)
{
    return v < lo ? lo : (v > hi ? hi : v);
}

void or_rct_forward(int32_t *c0, int32_t *c1, int32_t *c2, size_t n, int bits)
{
    const int32_t dc = 1 << (bits - 1);
    for (size_t i = 0; i < n; i++) {
        const int32_t r = c0[i] - dc, g = c1[i] - dc, b = c2[i] - dc;
        c0[i] = (r + 2 * g + b) >> 2;
        c1[i] = b - g;
        c2[i] = r - g;
    }
}

/* Output range of `bits` (OR_SIGNED set: signed samples, no DC level shift;
 * ISO G.1.2 shifts unsigned components only). */
static void out_range(int bits, int32_t *dc, int32_t *lo, int32_t *hi)
{
    const int b = bits & 0xFF;
    if (bits & OR_SIGNED) {
        *dc = 0;
        *lo = -(1 << (b - 1));
        *hi = (1 << (b - 1)) - 1;
    } else {
        *dc = 1 << (b - 1);
        *lo = 0;
        *hi = (1 << b) - 1;
    }
}

void or_rct_inverse(int32_t *c0, int32_t *c1, int32_t *c2, size_t n, int bits)
{
    int32_t dc, lo, mx;
    out_range(bits, &dc, &lo, &mx);
    for (size_t i = 0; i < n; i++) {
        const int32_t y = c0[i], u = c1[i], v = c2[i];
        const int32_t g = y - ((u + v) >> 2), r = v + g, b = u + g;
        c0[i] = clampi(r + dc, lo, mx);
        c1[i] = clampi(g + dc, lo, mx);
        c2[i] = clampi(b + dc, lo, mx);
    }
}

void or_ict_forward(const int32_t *r, const int32_t *g, const int32_t *b,
                    double *y, double *cb, double *cr, size_t n, int bits)
{
    const double dc = (double)(1 << (bits - 1));
    for (size_t i = 0; i < n; i++) {
        const double R = r[i] - dc, G = g[i] - dc, B = b[i] - dc;
        y[i] = 0.299 * R + 0.587 * G + 0.114 * B;
        cb[i] = -0.16875 * R - 0.33126 * G + 0.5 * B;
        cr[i] = 0.5 * R - 0.41869 * G - 0.08131 * B;
    }
}

void or_ict_inverse(const double *y, const double *cb, const double *cr,
                    int32_t *r, int32_t *g, int32_t *b, size_t n, int bits)
{
    int32_t dc, lo, mx;
    out_range(bits, &dc, &lo, &mx);
    for (size_t i = 0; i < n; i++) {
        const double R = y[i] + 1.402 * cr[i];
        const double G = y[i] - 0.34413 * cb[i] - 0.71414 * cr[i];
        const double B = y[i] + 1.772 * cb[i];
        r[i] = clampi((int32_t)rint(R) + dc, lo, mx);
        g[i] = clampi((int32_t)rint(G) + dc, lo, mx);
        b[i] = clampi((int32_t)rint(B) + dc, lo, mx);
    }
}

void or_dc_forward(int32_t *x, size_t n, int bits)
{
    for (size_t i = 0; i < n; i++) x[i] -= 1 << (bits - 1);
}

void or_dc_inverse_clamp(int32_t *x, size_t n, int bits)
{
    int32_t dc, lo, mx;
    out_range(bits, &dc, &lo, &mx);
    for (size_t i = 0; i < n; i++) x[i] = clampi(x[i] + dc, lo, mx);
}

void or_dc_inverse_float(const double *x, int32_t *out, size_t n, int bits)
{
    int32_t dc, lo, mx;
    out_range(bits, &dc, &lo, &mx);
    for (size_t i = 0; i < n; i++) out[i] = clampi((int32_t)rint(x[i]) + dc, lo, mx);
}

/* ===================== Whole-tile decode ================================= */

typedef struct {
    const or_cblk *cb;
    const uint8_t *pool;
    int w, h, ncomp, reversible;
    float r;
    int32_t *ip;
    double *fp;
    int err;
} or_t1_job;

static void or_t1_one(void *arg, int i)
{
    or_t1_job *J = (or_t1_job *)arg;
    const or_cblk *c = &J->cb[i];
    int32_t q[64 * 64];
    uint8_t u[64 * 64];
    const size_t np = (size_t)J->w * J->h;
    const int numbps = (int)c->mb - (int)c->zero_bitplanes;
    const int passes = numbps <= 0 ? 0 : c->passes;
    /* terminated segments: a table of their lengths precedes the codeword */
    uint32_t lens[256];
    int nseg = 0;
    const uint8_t *seg = J->pool + c->seg_off;
    if ((c->style & (OR_STYLE_BYPASS | OR_STYLE_TERMALL)) && passes > 0) {
        nseg = or_pass_segments(c->style, passes);
        for (int k = 0; k < nseg; k++)
            lens[k] = (uint32_t)seg[4 * k] | (uint32_t)seg[4 * k + 1] << 8 |
                      (uint32_t)seg[4 * k + 2] << 16 | (uint32_t)seg[4 * k + 3] << 24;
        seg += 4 * (size_t)nseg;
    }
    if (c->comp >= J->ncomp || c->out_x + c->w > (uint32_t)J->w || c->out_y + c->h > (uint32_t)J->h ||
        or_t1_decode_style(seg, (int)c->seg_len, c->w, c->h, c->orient, numbps < 0 ? 0 : numbps, passes,
                           c->style, nseg ? lens : NULL, nseg, q, u)) {
        __atomic_store_n(&J->err, 1, __ATOMIC_RELAXED);
        return;
    }
    /* ROI maxshift (ISO H.1): a magnitude >= 2^roi belongs to the region and
     * is scaled down by 2^roi, its undecoded planes with it; the background
     * keeps its value. */
    if (c->roi)
        for (int i = 0; i < c->w * c->h; i++) {
            const int32_t a = q[i] < 0 ? -q[i] : q[i];
            if (a >> c->roi) {
                q[i] = q[i] < 0 ? -(a >> c->roi) : (a >> c->roi);
                u[i] = (uint8_t)(u[i] > c->roi ? u[i] - c->roi : 0);
            }
        }
    for (int y = 0; y < c->h; y++) {
        const size_t o = (size_t)c->comp * np + (size_t)(c->out_y + y) * J->w + c->out_x;
        if (J->reversible) {
            or_dequant_int(q + y * c->w, u + y * c->w, c->w, J->r, J->ip + o);
        } else {
            float tmp[64];
            or_dequant_float(q + y * c->w, u + y * c->w, c->w, J->r, c->step, tmp);
            for (int x = 0; x < c->w; x++) J->fp[o + x] = tmp[x];
        }
    }
}

int or_decode_tile(const or_cblk *cb, int n, const uint8_t *pool,
                   int w, int h, int ncomp, int bits, int levels,
                   int reversible, int mct, float r, int threads,
                   uint16_t *out)
{
    return or_decode_tile_f64(cb, n, pool, w, h, ncomp, bits, levels, reversible, mct, r, threads, out, NULL);
}

int or_decode_tile_f64(const or_cblk *cb, int n, const uint8_t *pool,
                       int w, int h, int ncomp, int bits, int levels,
                       int reversible, int mct, float r, int threads,
                       uint16_t *out, double *out_f64)
{
    const size_t np = (size_t)w * h;
    int32_t *ip = NULL;
    double *fp = NULL;
    if (ncomp < 1 || ncomp > 4 || (bits & 0xFF) < 1 || (bits & 0xFF) > 16 || (bits & ~(0xFF | OR_SIGNED)) ||
        levels < 0 || levels > 32)
        return -1;
    if (reversible) ip = calloc(np * ncomp, sizeof(int32_t));
    else fp = calloc(np * ncomp, sizeof(double));
    if (!ip && !fp) return -2;
    {
        or_t1_job J = {cb, pool, w, h, ncomp, reversible, r, ip, fp, 0};
        or_parallel_for(n, threads, or_t1_one, &J);
        if (J.err) { free(ip); free(fp); return -3; }
    }
    for (int c = 0; c < ncomp; c++) {
        if (ip) idwt53_mt(ip + c * np, w, h, w, levels, OR_ROUND_FLOOR, threads);
        else idwt97_mt(fp + c * np, w, h, w, levels, threads);
    }
    if (reversible) {
        if (mct && ncomp >= 3) or_rct_inverse(ip, ip + np, ip + 2 * np, np, bits);
        else for (int c = 0; c < ncomp; c++) or_dc_inverse_clamp(ip + c * np, np, bits);
        if (mct && ncomp > 3) for (int c = 3; c < ncomp; c++) or_dc_inverse_clamp(ip + c * np, np, bits);
        for (size_t i = 0; i < np * ncomp; i++) out[i] = (uint16_t)ip[i];
    } else {
        int32_t *tmp = malloc(sizeof(int32_t) * np * ncomp);
        if (!tmp) { free(fp); return -2; }
        if (out_f64) {
            /* the unrounded samples: ISO G.2 inverse ICT, then the DC shift */
            int32_t dc, lo, mx;
            out_range(bits, &dc, &lo, &mx);
            for (int c = 0; c < ncomp; c++)
                for (size_t i = 0; i < np; i++) {
                    double v = fp[c * np + i];
                    if (mct && ncomp >= 3 && c < 3) {
                        const double y = fp[i], cb_ = fp[np + i], cr = fp[2 * np + i];
                        v = c == 0 ? y + 1.402 * cr : (c == 1 ? y - 0.34413 * cb_ - 0.71414 * cr : y + 1.772 * cb_);
                    }
                    out_f64[c * np + i] = v + dc;
                }
        }
        if (mct && ncomp >= 3) {
            or_ict_inverse(fp, fp + np, fp + 2 * np, tmp, tmp + np, tmp + 2 * np, np, bits);
            for (int c = 3; c < ncomp; c++) or_dc_inverse_float(fp + c * np, tmp + c * np, np, bits);
        } else {
            for (int c = 0; c < ncomp; c++) or_dc_inverse_float(fp + c * np, tmp + c * np, np, bits);
        }
        for (size_t i = 0; i < np * ncomp; i++) out[i] = (uint16_t)tmp[i];
        free(tmp);
    }
    free(ip);
    free(fp);
    return 0;
}

/* ===================== MQ encoder (ISO C.2) ============================== */
/* The reference decodes only and has no encoder; this restates the
 * normative encoder of ISO/IEC 15444-1 Annex C.2 (INITENC, CODEMPS,
 * CODELPS, RENORME, BYTEOUT, FLUSH) so that the oracle can generate its own
 * inputs.  The byte buffer keeps one byte in front of the codeword (the
 * "B[BPST-1]" of C.2.8), which starts at zero. */

typedef struct {
    uint8_t *buf;        /* buf[0] precedes the codeword */
    int cap, bp, ct, overflow;
    uint32_t a, c;
    uint8_t idx[NCX], mps[NCX];
} mqenc;

static void mqe_init(mqenc *e, uint8_t *buf, int cap)
{
    memset(e, 0, sizeof *e);
    e->buf = buf;
    e->cap = cap;
    e->buf[0] = 0;
    e->a = 0x8000;
    e->ct = 12;
    e->idx[0] = 4;          /* ISO Table D.7, as mq_reset */
    e->idx[CX_RUN] = 3;
    e->idx[CX_UNI] = 46;
}

static void mqe_put(mqenc *e, uint32_t v)
{
    e->bp++;
    if (e->bp < e->cap) e->buf[e->bp] = (uint8_t)v;
    else e->overflow = 1;
}

static uint32_t mqe_last(const mqenc *e) { return e->bp < e->cap ? e->buf[e->bp] : 0; }

/* BYTEOUT with bit stuffing after 0xFF and carry propagation into the
 * previous byte (ISO Figures C.8 and C.9). */
static void mqe_byteout(mqenc *e)
{
    if (mqe_last(e) == 0xFF) {
        mqe_put(e, e->c >> 20);
        e->c &= 0xFFFFF;
        e->ct = 7;
        return;
    }
    if (e->c < 0x8000000) {
        mqe_put(e, e->c >> 19);
        e->c &= 0x7FFFF;
        e->ct = 8;
        return;
    }
    if (e->bp < e->cap) e->buf[e->bp]++;
    if (mqe_last(e) == 0xFF) {
        e->c &= 0x7FFFFFF;
        mqe_put(e, e->c >> 20);
        e->c &= 0xFFFFF;
        e->ct = 7;
    } else {
        mqe_put(e, e->c >> 19);
        e->c &= 0x7FFFF;
        e->ct = 8;
    }
}

static void mqe_renorm(mqenc *e)
{
    do {
        e->a <<= 1;
        e->c <<= 1;
        if (--e->ct == 0) mqe_byteout(e);
    } while ((e->a & 0x8000) == 0);
}

/* ENCODE (ISO Figure C.3): CODEMPS / CODELPS with conditional exchange. */
static void mqe_encode(mqenc *e, int d, int cx)
{
    const int s = e->idx[cx];
    const uint32_t qe = kQe[s];
    e->a -= qe;
    if (d == e->mps[cx]) {
        if (e->a & 0x8000) {
            e->c += qe;
            return;
        }
        if (e->a < qe) e->a = qe;
        else e->c += qe;
        e->idx[cx] = kNMPS[s];
    } else {
        if (e->a < qe) e->c += qe;
        else e->a = qe;
        if (kSWITCH[s]) e->mps[cx] ^= 1;
        e->idx[cx] = kNLPS[s];
    }
    mqe_renorm(e);
}

/* FLUSH with SETBITS (ISO Figures C.11-C.12); a final 0xFF is dropped.
 * Returns the codeword length. */
static int mqe_flush(mqenc *e)
{
    const uint32_t tempc = e->c + e->a;
    e->c |= 0xFFFF;
    if (e->c >= tempc) e->c -= 0x8000;
    e->c <<= e->ct;
    mqe_byteout(e);
    e->c <<= e->ct;
    mqe_byteout(e);
    return mqe_last(e) == 0xFF ? e->bp - 1 : e->bp;
}

/* ===================== Tier-1 encoder (ISO D) ============================ */
/* The mirror of the passes above: each decision the decoder reads is the
 * bit the encoder writes with the same context, in the same scan order. */

static void encode_sign(mqenc *e, const t1st *s, int x, int y, int neg)
{
    int hc, vc, cx, xr;
#define CONTRIB(xx, yy) (AT(s, sig, xx, yy) ? (AT(s, sgn, xx, yy) ? -1 : 1) : 0)
    hc = CONTRIB(x - 1, y) + CONTRIB(x + 1, y);
    vc = CONTRIB(x, y - 1) + CONTRIB(x, y + 1);
#undef CONTRIB
    hc = hc > 1 ? 1 : (hc < -1 ? -1 : hc);
    vc = vc > 1 ? 1 : (vc < -1 ? -1 : vc);
    if (hc == 0) {
        cx = vc == 0 ? 9 : 10;
        xr = vc < 0;
    } else {
        cx = 12 + hc * vc;
        xr = hc < 0;
    }
    mqe_encode(e, neg ^ xr, cx);
}

static void enc_significant(mqenc *e, t1st *s, const int32_t *coef, int x, int y)
{
    const int neg = coef[y * s->w + x] < 0;
    encode_sign(e, s, x, y, neg);
    AT(s, sgn, x, y) = (uint8_t)neg;
    AT(s, sig, x, y) = 1;
}

static inline int mag_bit(const int32_t *coef, int w, int x, int y, int p)
{
    const int32_t v = coef[y * w + x];
    return (int)(((uint32_t)(v < 0 ? -v : v) >> p) & 1u);
}

static void enc_spp(mqenc *e, t1st *s, const int32_t *coef, int orient, int p)
{
    for (int y0 = 0; y0 < s->h; y0 += 4)
        for (int x = 0; x < s->w; x++)
            for (int y = y0; y < y0 + 4 && y < s->h; y++) {
                int hh, vv, dd, b;
                if (AT(s, sig, x, y)) continue;
                nb_counts(s, x, y, &hh, &vv, &dd);
                if (hh + vv + dd == 0) continue;
                AT(s, vis, x, y) = 1;
                b = mag_bit(coef, s->w, x, y, p);
                mqe_encode(e, b, zc_context(orient, hh, vv, dd));
                if (b) enc_significant(e, s, coef, x, y);
            }
}

static void enc_mrp(mqenc *e, t1st *s, const int32_t *coef, int p)
{
    for (int y0 = 0; y0 < s->h; y0 += 4)
        for (int x = 0; x < s->w; x++)
            for (int y = y0; y < y0 + 4 && y < s->h; y++) {
                int hh, vv, dd;
                if (!AT(s, sig, x, y) || AT(s, vis, x, y)) continue;
                nb_counts(s, x, y, &hh, &vv, &dd);
                mqe_encode(e, mag_bit(coef, s->w, x, y, p), AT(s, ref, x, y) ? 16 : (hh + vv + dd ? 15 : 14));
                AT(s, ref, x, y) = 1;
            }
}

static void enc_cup(mqenc *e, t1st *s, const int32_t *coef, int orient, int p)
{
    for (int y0 = 0; y0 < s->h; y0 += 4)
        for (int x = 0; x < s->w; x++) {
            int y = y0;
            if (y0 + 4 <= s->h) {
                int ok = 1;
                for (int k = 0; k < 4 && ok; k++) {
                    int hh, vv, dd;
                    if (AT(s, sig, x, y0 + k) || AT(s, vis, x, y0 + k)) { ok = 0; break; }
                    nb_counts(s, x, y0 + k, &hh, &vv, &dd);
                    if (hh + vv + dd) ok = 0;
                }
                if (ok) {
                    int r = 0;
                    while (r < 4 && !mag_bit(coef, s->w, x, y0 + r, p)) r++;
                    if (r == 4) {
                        mqe_encode(e, 0, CX_RUN);
                        continue;
                    }
                    mqe_encode(e, 1, CX_RUN);
                    mqe_encode(e, r >> 1, CX_UNI);
                    mqe_encode(e, r & 1, CX_UNI);
                    enc_significant(e, s, coef, x, y0 + r);
                    y = y0 + r + 1;
                }
            }
            for (; y < y0 + 4 && y < s->h; y++) {
                int hh, vv, dd, b;
                if (AT(s, sig, x, y) || AT(s, vis, x, y)) continue;
                nb_counts(s, x, y, &hh, &vv, &dd);
                b = mag_bit(coef, s->w, x, y, p);
                mqe_encode(e, b, zc_context(orient, hh, vv, dd));
                if (b) enc_significant(e, s, coef, x, y);
            }
        }
}

int or_t1_encode(const int32_t *coef, int w, int h, int orient, int passes,
                 uint8_t *out, int cap, int *len, int *passes_out, int *numbps_out)
{
    t1st st;
    mqenc e;
    uint32_t mx = 0;
    int numbps = 0, total, pi = 0;
    uint8_t *buf;
    if (!coef || !out || !len || w < 1 || h < 1 || w > 64 || h > 64 || orient < 0 || orient > 3 || cap < 0)
        return -1;
    for (int i = 0; i < w * h; i++) {
        const uint32_t a = (uint32_t)(coef[i] < 0 ? -coef[i] : coef[i]);
        if (a > mx) mx = a;
    }
    while (numbps < 31 && (mx >> numbps)) numbps++;
    if (mx >> numbps) return -1;   /* magnitude needs more than 31 bit-planes */
    total = numbps ? 3 * numbps - 2 : 0;
    if (passes <= 0 || passes > total) passes = total;
    if (passes_out) *passes_out = passes;
    if (numbps_out) *numbps_out = numbps;
    *len = 0;
    if (passes == 0) return 0;
    if (t1_alloc(&st, w, h)) { t1_free(&st); return -2; }
    st.vsc = 0;
    buf = malloc((size_t)cap + 1);
    if (!buf) { t1_free(&st); return -2; }
    mqe_init(&e, buf, cap + 1);
    for (int p = numbps - 1; p >= 0 && pi < passes; p--) {
        if (p != numbps - 1) {
            enc_spp(&e, &st, coef, orient, p);
            if (++pi >= passes) break;
            enc_mrp(&e, &st, coef, p);
            if (++pi >= passes) break;
        }
        enc_cup(&e, &st, coef, orient, p);
        ++pi;
        memset(st.vis, 0, (size_t)st.W * (st.h + 2));
    }
    *len = mqe_flush(&e);
    t1_free(&st);
    if (e.overflow || *len > cap) { free(buf); return -3; }
    memcpy(out, buf + 1, (size_t)*len);
    free(buf);
    return 0;
}

/* ===================== Whole-tile encode ================================= */
/* The forward pipeline the bench workloads are coded with: DC level shift,
 * forward RCT or ICT (preprocess_rct.cl:18-31, preprocess_ict.cl:20-37),
 * multi-level forward 5/3 or 9/7 (dwt_f53.cl, dwt_f97.cl; ISO F.4),
 * deadzone quantisation with the step of ISO E.1 derived from a base step
 * scaled by the band's synthesis L2 norm and rounded to its (exponent,
 * mantissa) code, and Tier-1 per code-block with every pass kept. */

/* log2 of the nominal gain of a band: 0 LL, 1 HL/LH, 2 HH (ISO E.1.1.1). */
static int band_gain(int orient) { return orient == 0 ? 0 : (orient == 3 ? 2 : 1); }

/* The step a decoder derives from the (exponent, mantissa) pair that codes
 * delta for a band with rb = bits + gain (ISO E.1, Equation E-3). */
static double coded_step(double delta, int rb)
{
    int ex = rb - (int)floor(log2(delta));
    int mu = (int)lround((delta / ldexp(1.0, rb - ex) - 1.0) * 2048.0);
    if (mu >= 2048) { mu = 0; ex--; }
    if (mu < 0) mu = 0;
    return ldexp(1.0 + mu / 2048.0, rb - ex);
}

typedef struct {
    int comp, orient, level, x0, y0, w, h;
    double step;
} or_band;

typedef struct {
    const or_band *band;
    int bx, by;           /* block position inside the band */
} or_blockjob;

typedef struct {
    const or_blockjob *jobs;
    const int32_t *q;     /* quantised planes, ncomp * w * h */
    int w, h, cblk;
    uint8_t **words;
    or_cblk *cb;
    int err;
} or_enc_job;

static void or_enc_one(void *arg, int k)
{
    or_enc_job *J = (or_enc_job *)arg;
    const or_blockjob *jb = &J->jobs[k];
    const or_band *b = jb->band;
    const int bw = (b->w - jb->bx) < J->cblk ? (b->w - jb->bx) : J->cblk;
    const int bh = (b->h - jb->by) < J->cblk ? (b->h - jb->by) : J->cblk;
    const int cap = 8 * bw * bh + 64;
    int32_t blk[64 * 64];
    int len = 0, passes = 0, numbps = 0;
    const size_t plane = (size_t)J->w * J->h;
    or_cblk *c = &J->cb[k];
    for (int y = 0; y < bh; y++)
        for (int x = 0; x < bw; x++)
            blk[y * bw + x] = J->q[(size_t)b->comp * plane + (size_t)(b->y0 + jb->by + y) * J->w + b->x0 + jb->bx + x];
    J->words[k] = malloc((size_t)cap);
    if (!J->words[k] || or_t1_encode(blk, bw, bh, b->orient, 0, J->words[k], cap, &len, &passes, &numbps)) {
        __atomic_store_n(&J->err, 1, __ATOMIC_RELAXED);
        return;
    }
    memset(c, 0, sizeof *c);
    c->seg_len = (uint32_t)len;
    c->w = (uint16_t)bw;
    c->h = (uint16_t)bh;
    c->passes = (uint8_t)passes;
    c->mb = 31;
    c->zero_bitplanes = (uint8_t)(31 - numbps);
    c->orient = (uint8_t)b->orient;
    c->comp = (uint8_t)b->comp;
    c->out_x = (uint32_t)(b->x0 + jb->bx);
    c->out_y = (uint32_t)(b->y0 + jb->by);
    c->step = (float)b->step;
}

int or_encode_tile(const uint16_t *samples, int w, int h, int ncomp, int bits,
                   int levels, int reversible, int mct, double base_step, int cblk,
                   int threads, or_cblk **cb_out, int *n_out, uint8_t **pool_out,
                   size_t *pool_len_out)
{
    const size_t np = (size_t)w * h;
    const int usemct = mct && ncomp >= 3;
    const int32_t dc = 1 << (bits - 1);
    int32_t *q = NULL;
    double *fp = NULL;
    or_band bands[4 * (3 * 32 + 1)];
    int nb = 0, nj = 0, lw[34], lh[34];
    or_blockjob *jobs = NULL;
    or_cblk *cb = NULL;
    uint8_t **words = NULL, *pool = NULL;
    size_t total = 0;
    int rc = 0;
    if (!samples || !cb_out || !n_out || !pool_out || !pool_len_out || w < 1 || h < 1 || ncomp < 1 ||
        ncomp > 4 || bits < 1 || bits > 16 || levels < 0 || levels > 32 || cblk < 4 || cblk > 64 ||
        (cblk & (cblk - 1)) || (!reversible && !(base_step > 0.0)))
        return -1;
    q = malloc(sizeof(int32_t) * np * ncomp);
    if (!q) return -2;
    for (size_t i = 0; i < np * ncomp; i++) q[i] = (int32_t)samples[i] - dc;
    if (reversible) {
        if (usemct)
            for (size_t i = 0; i < np; i++) {
                const int32_t r = q[i], g = q[np + i], b = q[2 * np + i];
                q[i] = (r + 2 * g + b) >> 2;   /* ISO G.2: floor */
                q[np + i] = b - g;
                q[2 * np + i] = r - g;
            }
        for (int c = 0; c < ncomp; c++) fdwt53_mt(q + c * np, w, h, w, levels, OR_ROUND_FLOOR, threads);
    } else {
        fp = malloc(sizeof(double) * np * ncomp);
        if (!fp) { free(q); return -2; }
        for (size_t i = 0; i < np * ncomp; i++) fp[i] = (double)q[i];
        if (usemct)
            for (size_t i = 0; i < np; i++) {
                const double R = fp[i], G = fp[np + i], B = fp[2 * np + i];
                fp[i] = 0.299 * R + 0.587 * G + 0.114 * B;
                fp[np + i] = -0.16875 * R - 0.33126 * G + 0.5 * B;
                fp[2 * np + i] = 0.5 * R - 0.41869 * G - 0.08131 * B;
            }
        for (int c = 0; c < ncomp; c++) fdwt97_mt(fp + c * np, w, h, w, levels, threads);
    }
    /* band geometry of the Mallat plane (ISO B.5, a tile at the origin) */
    lw[0] = w; lh[0] = h;
    for (int l = 1; l <= levels; l++) { lw[l] = (lw[l - 1] + 1) / 2; lh[l] = (lh[l - 1] + 1) / 2; }
    for (int c = 0; c < ncomp; c++) {
        bands[nb++] = (or_band){c, 0, levels, 0, 0, lw[levels], lh[levels], 1.0};
        for (int l = levels; l >= 1; l--)
            for (int o = 1; o <= 3; o++)
                bands[nb++] = (or_band){c, o, l, (o & 1) ? lw[l] : 0, (o & 2) ? lh[l] : 0,
                                        (o & 1) ? lw[l - 1] - lw[l] : lw[l], (o & 2) ? lh[l - 1] - lh[l] : lh[l],
                                        1.0};
    }
    for (int k = 0; k < nb; k++) {
        or_band *b = &bands[k];
        if (!reversible)
            b->step = coded_step(base_step * ldexp(1.0, bits) / or_subband_norm(1, b->level, b->orient),
                                 bits + band_gain(b->orient));
        if (b->w > 0 && b->h > 0) nj += ((b->w + cblk - 1) / cblk) * ((b->h + cblk - 1) / cblk);
    }
    /* deadzone quantisation (ISO E.1: q = sign(y) floor(|y| / step)) */
    if (!reversible)
        for (int k = 0; k < nb; k++) {
            const or_band *b = &bands[k];
            for (int y = b->y0; y < b->y0 + b->h; y++)
                for (int x = b->x0; x < b->x0 + b->w; x++) {
                    const size_t i = (size_t)b->comp * np + (size_t)y * w + x;
                    const int32_t v = (int32_t)floor(fabs(fp[i]) / b->step);
                    q[i] = fp[i] < 0 ? -v : v;
                }
        }
    free(fp);
    jobs = malloc(sizeof(or_blockjob) * (nj ? nj : 1));
    cb = calloc(nj ? nj : 1, sizeof(or_cblk));
    words = calloc(nj ? nj : 1, sizeof(uint8_t *));
    if (!jobs || !cb || !words) { rc = -2; goto done; }
    nj = 0;
    for (int k = 0; k < nb; k++)
        for (int by = 0; by < bands[k].h; by += cblk)
            for (int bx = 0; bx < bands[k].w; bx += cblk) jobs[nj++] = (or_blockjob){&bands[k], bx, by};
    {
        or_enc_job J = {jobs, q, w, h, cblk, words, cb, 0};
        or_parallel_for(nj, threads, or_enc_one, &J);
        if (J.err) { rc = -3; goto done; }
    }
    /* segment pool: codewords one after the other, 16-byte aligned */
    for (int k = 0; k < nj; k++) total += (cb[k].seg_len + 15u) & ~(size_t)15u;
    pool = calloc(total ? total : 16, 1);
    if (!pool) { rc = -2; goto done; }
    total = 0;
    for (int k = 0; k < nj; k++) {
        cb[k].seg_off = total;
        memcpy(pool + total, words[k], cb[k].seg_len);
        total += (cb[k].seg_len + 15u) & ~(size_t)15u;
    }
    *cb_out = cb;
    *n_out = nj;
    *pool_out = pool;
    *pool_len_out = total;
    cb = NULL;
done:
    if (words)
        for (int k = 0; k < nj; k++) free(words[k]);
    free(words);
    free(jobs);
    free(cb);
    free(q);
    return rc;
}

void or_encoded_free(or_cblk *cb, uint8_t *pool)
{
    free(cb);
    free(pool);
}

/* ===================== Truncated coefficients (ISO D.3, E.1.1.2) ========= */
/* What a decoder reconstructs from the first `passes` coding passes of a
 * block, computed from the coefficients themselves and the pass structure
 * of ISO D.3, without any MQ coding: every coefficient is coded once per
 * bit-plane, so after complete bit-planes it is known down to the last
 * one.  In a bit-plane cut after its significance-propagation pass only the
 * coefficients that pass visited (insignificant, with a significant
 * neighbour at their turn in the scan, ISO D.3.1) carry that plane; cut
 * after the refinement pass, the coefficients significant before the plane
 * carry it too (ISO D.3.3).  The value keeps the known bits; the sign
 * counts once the value is non-zero. */
void or_t1_truncate(const int32_t *coef, int w, int h, int passes, int32_t *out)
{
    uint32_t mx = 0;
    int nb = 0, total, t, plane, type;
    for (int i = 0; i < w * h; i++) {
        const uint32_t a = (uint32_t)(coef[i] < 0 ? -coef[i] : coef[i]);
        if (a > mx) mx = a;
    }
    while (nb < 31 && (mx >> nb)) nb++;
    total = nb ? 3 * nb - 2 : 0;
    if (passes <= 0) {
        for (int i = 0; i < w * h; i++) out[i] = 0;
        return;
    }
    if (passes >= total) {
        for (int i = 0; i < w * h; i++) out[i] = coef[i];
        return;
    }
    t = passes - 1;                       /* the last pass kept */
    plane = t == 0 ? nb - 1 : nb - 1 - (t + 2) / 3;
    type = t == 0 ? 2 : (t - 1) % 3;      /* 0 SPP, 1 MRP, 2 cleanup */
    {
        /* low[i]: lowest plane known; 1 + plane unless the cut pass coded it */
        uint8_t *low = malloc((size_t)w * h), *sig = calloc((size_t)(w + 2) * (h + 2), 1);
        const int W = w + 2;
#define SIG(x, y) sig[((y) + 1) * W + (x) + 1]
        for (int i = 0; i < w * h; i++) low[i] = (uint8_t)(type == 2 ? plane : plane + 1);
        if (type != 2) {
            for (int y = 0; y < h; y++)
                for (int x = 0; x < w; x++) {
                    const int32_t v = coef[y * w + x];
                    SIG(x, y) = (((uint32_t)(v < 0 ? -v : v)) >> (plane + 1)) != 0;
                    if (type == 1 && SIG(x, y)) low[y * w + x] = (uint8_t)plane;
                }
            for (int y0 = 0; y0 < h; y0 += 4)
                for (int x = 0; x < w; x++)
                    for (int y = y0; y < y0 + 4 && y < h; y++) {
                        int n;
                        const int32_t v = coef[y * w + x];
                        if (SIG(x, y)) continue;
                        n = SIG(x - 1, y - 1) + SIG(x, y - 1) + SIG(x + 1, y - 1) + SIG(x - 1, y) + SIG(x + 1, y) +
                            SIG(x - 1, y + 1) + SIG(x, y + 1) + SIG(x + 1, y + 1);
                        if (!n) continue;
                        low[y * w + x] = (uint8_t)plane;
                        if ((((uint32_t)(v < 0 ? -v : v)) >> plane) & 1u) SIG(x, y) = 1;
                    }
        }
#undef SIG
        for (int i = 0; i < w * h; i++) {
            const uint32_t a = (uint32_t)(coef[i] < 0 ? -coef[i] : coef[i]);
            const int32_t k = (int32_t)((a >> low[i]) << low[i]);
            out[i] = coef[i] < 0 ? -k : k;
        }
        free(low);
        free(sig);
    }
}

typedef struct {
    const int32_t *coef;
    const uint64_t *off;
    const uint16_t *w, *h;
    const uint8_t *passes;
    int32_t *out;
} or_trunc_job;

static void or_trunc_one(void *arg, int i)
{
    const or_trunc_job *J = (const or_trunc_job *)arg;
    or_t1_truncate(J->coef + J->off[i], J->w[i], J->h[i], J->passes[i], J->out + J->off[i]);
}

void or_t1_truncate_batch(const int32_t *coef, const uint64_t *off, const uint16_t *w, const uint16_t *h,
                          const uint8_t *passes, int n, int threads, int32_t *out)
{
    or_trunc_job J = {coef, off, w, h, passes, out};
    or_parallel_for(n, threads, or_trunc_one, &J);
}
