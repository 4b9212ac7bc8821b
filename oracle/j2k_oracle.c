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

/* Generic level driver over a strided line: gather -> (de)interleave ->
 * 1-D transform -> scatter.  ELEM/FN choose the sample type and filter. */
#define DEFINE_LEVEL(NAME, T, BODY_FWD)                                        \
    static void NAME(T *x, int w, int h, int pitch, int fwd, int rnd)          \
    {                                                                          \
        const int nmax = w > h ? w : h;                                        \
        T *line = malloc(sizeof(T) * nmax), *tmp = malloc(sizeof(T) * nmax);   \
        (void)rnd;                                                             \
        for (int pass = 0; pass < 2; pass++) {                                 \
            /* forward: columns then rows; reverse: rows then columns */       \
            const int vertical = fwd ? (pass == 0) : (pass == 1);              \
            const int n = vertical ? h : w, lines = vertical ? w : h;          \
            const int nl = (n + 1) / 2;                                        \
            for (int l = 0; l < lines; l++) {                                  \
                T *base = vertical ? x + l : x + (size_t)l * pitch;            \
                const size_t step = vertical ? (size_t)pitch : 1;              \
                for (int i = 0; i < n; i++) line[i] = base[i * step];          \
                if (fwd) {                                                     \
                    BODY_FWD(line, n, 1);                                      \
                    for (int i = 0; i < n; i++)                                \
                        tmp[(i & 1) ? nl + i / 2 : i / 2] = line[i];           \
                } else {                                                       \
                    for (int i = 0; i < n; i++)                                \
                        tmp[i] = line[(i & 1) ? nl + i / 2 : i / 2];           \
                    BODY_FWD(tmp, n, 0);                                       \
                }                                                              \
                for (int i = 0; i < n; i++) base[i * step] = tmp[i];           \
            }                                                                  \
        }                                                                      \
        free(line);                                                            \
        free(tmp);                                                             \
    }

#define F53(v, n, fwd) do { if (fwd) fdwt53_1d(v, n, rnd); else idwt53_1d(v, n, rnd); } while (0)
#define F97(v, n, fwd) do { if (fwd) fdwt97_1d(v, n); else idwt97_1d(v, n); } while (0)
DEFINE_LEVEL(level53, int32_t, F53)
DEFINE_LEVEL(level97, double, F97)

void or_fdwt53(int32_t *x, int w, int h, int pitch, int levels, int rounding)
{
    for (int l = 0; l < levels; l++) {
        level53(x, w, h, pitch, 1, rounding);
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
}

void or_idwt53(int32_t *x, int w, int h, int pitch, int levels, int rounding)
{
    int ws[33], hs[33];
    ws[0] = w; hs[0] = h;
    for (int l = 1; l <= levels; l++) { ws[l] = (ws[l - 1] + 1) / 2; hs[l] = (hs[l - 1] + 1) / 2; }
    for (int l = levels - 1; l >= 0; l--) level53(x, ws[l], hs[l], pitch, 0, rounding);
}

void or_fdwt97(double *x, int w, int h, int pitch, int levels)
{
    for (int l = 0; l < levels; l++) {
        level97(x, w, h, pitch, 1, 0);
        w = (w + 1) / 2;
        h = (h + 1) / 2;
    }
}

void or_idwt97(double *x, int w, int h, int pitch, int levels)
{
    int ws[33], hs[33];
    ws[0] = w; hs[0] = h;
    for (int l = 1; l <= levels; l++) { ws[l] = (ws[l - 1] + 1) / 2; hs[l] = (hs[l - 1] + 1) / 2; }
    for (int l = levels - 1; l >= 0; l--) level97(x, ws[l], hs[l], pitch, 0, 0);
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

typedef struct {
    int32_t *ip;
    double *fp;
    int w, h, levels;
} or_dwt_job;

static void or_dwt_one(void *arg, int c)
{
    or_dwt_job *J = (or_dwt_job *)arg;
    const size_t np = (size_t)J->w * J->h;
    if (J->ip) or_idwt53(J->ip + c * np, J->w, J->h, J->w, J->levels, OR_ROUND_FLOOR);
    else or_idwt97(J->fp + c * np, J->w, J->h, J->w, J->levels);
}

int or_decode_tile(const or_cblk *cb, int n, const uint8_t *pool,
                   int w, int h, int ncomp, int bits, int levels,
                   int reversible, int mct, float r, int threads,
                   uint16_t *out)
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
    {
        or_dwt_job D = {ip, fp, w, h, levels};
        or_parallel_for(ncomp, threads, or_dwt_one, &D);
    }
    if (reversible) {
        if (mct && ncomp >= 3) or_rct_inverse(ip, ip + np, ip + 2 * np, np, bits);
        else for (int c = 0; c < ncomp; c++) or_dc_inverse_clamp(ip + c * np, np, bits);
        if (mct && ncomp > 3) for (int c = 3; c < ncomp; c++) or_dc_inverse_clamp(ip + c * np, np, bits);
        for (size_t i = 0; i < np * ncomp; i++) out[i] = (uint16_t)ip[i];
    } else {
        int32_t *tmp = malloc(sizeof(int32_t) * np * ncomp);
        if (!tmp) { free(fp); return -2; }
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
