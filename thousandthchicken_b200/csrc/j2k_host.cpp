// j2k_host.cpp -- host-side JPEG 2000 codestream handling for the B200 decode
// pipeline:
//   * geometry of resolutions / subbands / code-blocks (ISO B.5-B.7),
//   * the Tier-2 parser that turns a codestream into tc_cblk_desc records
//     (the hand-off the reference makes through codeBlockCallback,
//     codestream.c:336-470),
//   * the harness encoder used to generate test and benchmark codestreams:
//     forward colour transform + DWT on the CPU, deadzone quantisation, an
//     MQ/EBCOT Tier-1 encoder and a single-tile packet writer.
// The encoder exists because the reference ships no encoder and no sample
// files; it writes the subset the parser reads (one tile, one precinct per
// resolution, code-block style 0).
#include "j2k_host.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>

namespace tc {

// ============================ small utilities ================================

static int hw_threads(int req)
{
    if (req > 0) return req;
    unsigned n = std::thread::hardware_concurrency();
    return n ? (int)n : 1;
}

static void parallel_for(int n, int threads, const std::function<void(int)> &fn)
{
    threads = std::min(hw_threads(threads), std::max(n, 1));
    if (threads <= 1) {
        for (int i = 0; i < n; i++) fn(i);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
        pool.emplace_back([&] {
            for (int i; (i = next.fetch_add(1)) < n;) fn(i);
        });
    for (auto &th : pool) th.join();
}

static inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

// ============================ geometry ======================================

void level_sizes(int w, int h, int levels, std::vector<int> &ws, std::vector<int> &hs)
{
    ws.assign(levels + 1, 0);
    hs.assign(levels + 1, 0);
    ws[0] = w;
    hs[0] = h;
    for (int d = 1; d <= levels; d++) {
        ws[d] = (ws[d - 1] + 1) / 2;
        hs[d] = (hs[d - 1] + 1) / 2;
    }
}

std::vector<Resolution> make_geometry(int w, int h, int levels, int xcb, int ycb)
{
    std::vector<int> ws, hs;
    level_sizes(w, h, levels, ws, hs);
    std::vector<Resolution> res(levels + 1);
    auto finish = [&](Band &b) {
        b.cbw_log2 = xcb;
        b.cbh_log2 = ycb;
        b.ncbx = b.w > 0 ? ceil_div(b.w, 1 << xcb) : 0;
        b.ncby = b.h > 0 ? ceil_div(b.h, 1 << ycb) : 0;
    };
    Band ll;
    ll.orient = 0;
    ll.level = levels;
    ll.w = ws[levels];
    ll.h = hs[levels];
    finish(ll);
    res[0].w = ws[levels];
    res[0].h = hs[levels];
    res[0].bands.push_back(ll);
    for (int r = 1; r <= levels; r++) {
        const int d = levels - r + 1;
        res[r].w = ws[d - 1];
        res[r].h = hs[d - 1];
        for (int o = 1; o <= 3; o++) {
            Band b;
            b.orient = o;
            b.level = d;
            b.x0 = (o & 1) ? ws[d] : 0;
            b.y0 = (o & 2) ? hs[d] : 0;
            b.w = (o & 1) ? ws[d - 1] - ws[d] : ws[d];
            b.h = (o & 2) ? hs[d - 1] - hs[d] : hs[d];
            finish(b);
            res[r].bands.push_back(b);
        }
    }
    return res;
}

// ============================ DWT (CPU, encoder side) =======================

static inline int pse(int i, int n)
{
    if (n == 1) return 0;
    const int per = 2 * (n - 1);
    i %= per;
    if (i < 0) i += per;
    return i >= n ? per - i : i;
}

static inline int32_t floordiv(int32_t a, int b)
{
    int32_t q = a / b;
    if ((a % b) != 0 && ((a < 0) != (b < 0))) q--;
    return q;
}

static const double kA = -1.586134342059924, kB = -0.052980118572961,
                    kG = 0.882911075530934, kD = 0.443506852043971,
                    kK = 1.230174104914001;

static void fwd53_line(int32_t *x, int n)
{
    if (n < 2) return;
    for (int k = 1; k < n; k += 2) x[k] -= floordiv(x[pse(k - 1, n)] + x[pse(k + 1, n)], 2);
    for (int k = 0; k < n; k += 2) x[k] += floordiv(x[pse(k - 1, n)] + x[pse(k + 1, n)] + 2, 4);
}

static void fwd97_line(double *x, int n)
{
    if (n < 2) return;
    for (int k = 1; k < n; k += 2) x[k] += kA * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 0; k < n; k += 2) x[k] += kB * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 1; k < n; k += 2) x[k] += kG * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 0; k < n; k += 2) x[k] += kD * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 1; k < n; k += 2) x[k] *= kK;
    for (int k = 0; k < n; k += 2) x[k] *= 1.0 / kK;
}

static void inv97_line(double *x, int n)
{
    if (n < 2) return;
    for (int k = 0; k < n; k += 2) x[k] *= kK;
    for (int k = 1; k < n; k += 2) x[k] *= 1.0 / kK;
    for (int k = 0; k < n; k += 2) x[k] -= kD * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 1; k < n; k += 2) x[k] -= kG * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 0; k < n; k += 2) x[k] -= kB * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 1; k < n; k += 2) x[k] -= kA * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
}

static void inv53r_line(double *x, int n)
{
    if (n < 2) return;
    for (int k = 0; k < n; k += 2) x[k] -= 0.25 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
    for (int k = 1; k < n; k += 2) x[k] += 0.5 * (x[pse(k - 1, n)] + x[pse(k + 1, n)]);
}

// Forward multi-level transform on a plane (vertical then horizontal per
// level, ISO F.4.2), output in Mallat layout.
template <typename T, typename F>
static void fwd_plane_pitch(T *x, int w, int h, size_t pitch, int levels, F line_fn, int threads)
{
    for (int l = 0; l < levels; l++) {
        const int nl_h = (h + 1) / 2, nl_w = (w + 1) / 2;
        // vertical
        const int cgroups = ceil_div(w, 16);
        parallel_for(cgroups, threads, [&](int g) {
            std::vector<T> a(h), b(h);
            for (int c = g * 16; c < std::min(w, g * 16 + 16); c++) {
                for (int i = 0; i < h; i++) a[i] = x[(size_t)i * pitch + c];
                line_fn(a.data(), h);
                for (int i = 0; i < h; i++) b[(i & 1) ? nl_h + i / 2 : i / 2] = a[i];
                for (int i = 0; i < h; i++) x[(size_t)i * pitch + c] = b[i];
            }
        });
        // horizontal
        parallel_for(h, threads, [&](int r) {
            std::vector<T> a(w);
            T *row = x + (size_t)r * pitch;
            for (int i = 0; i < w; i++) a[i] = row[i];
            line_fn(a.data(), w);
            for (int i = 0; i < w; i++) row[(i & 1) ? nl_w + i / 2 : i / 2] = a[i];
        });
        w = nl_w;
        h = nl_h;
    }
}

double subband_norm(bool wavelet97, int level, int orient)
{
    auto norm1d = [&](int lvl, int high) {
        const int n = 1 << (lvl + 7);
        std::vector<double> x(n, 0.0), t(n);
        int len = n;
        for (int l = 0; l < lvl; l++) len = (len + 1) / 2;
        x[high ? len + len / 2 : len / 2] = 1.0;
        for (int l = lvl - 1; l >= 0; l--) {
            int m = n;
            for (int k = 0; k < l; k++) m = (m + 1) / 2;
            for (int i = 0; i < m; i++) t[i] = x[(i & 1) ? (m + 1) / 2 + i / 2 : i / 2];
            if (wavelet97) inv97_line(t.data(), m);
            else inv53r_line(t.data(), m);
            std::copy(t.begin(), t.begin() + m, x.begin());
        }
        double s = 0.0;
        for (double v : x) s += v * v;
        return std::sqrt(s);
    };
    const double lo = norm1d(level, 0), hi = norm1d(level, 1);
    switch (orient) {
    case 0: return lo * lo;
    case 1: return hi * lo;
    case 2: return lo * hi;
    default: return hi * hi;
    }
}

// ============================ MQ encoder (ISO C.2) ==========================

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
static const uint8_t kSW[47] = {1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0};

struct MQEnc {
    std::vector<uint8_t> buf;  // buf[0] is the byte before the codeword
    size_t bp = 0;
    uint32_t a = 0x8000, c = 0;
    int ct = 12;
    uint8_t idx[19]{}, mps[19]{};

    MQEnc()
    {
        buf.reserve(4096);
        buf.push_back(0);
        reset_contexts();
    }
    // Initial probability states (ISO Table D.7).
    void reset_contexts()
    {
        for (int i = 0; i < 19; i++) idx[i] = mps[i] = 0;
        idx[0] = 4;
        idx[18] = 3;
        idx[17] = 46;
    }
    // A new codeword segment (after a termination): the coder registers
    // start over, the contexts carry on.
    void restart()
    {
        buf.assign(1, 0);
        bp = 0;
        a = 0x8000;
        c = 0;
        ct = 12;
    }
    void put(uint32_t v)
    {
        bp++;
        if (bp >= buf.size()) buf.push_back((uint8_t)v);
        else buf[bp] = (uint8_t)v;
    }
    void byteout()
    {
        if (buf[bp] == 0xFF) {
            put(c >> 20);
            c &= 0xFFFFF;
            ct = 7;
        } else if (c < 0x8000000) {
            put(c >> 19);
            c &= 0x7FFFF;
            ct = 8;
        } else {
            buf[bp]++;
            if (buf[bp] == 0xFF) {
                c &= 0x7FFFFFF;
                put(c >> 20);
                c &= 0xFFFFF;
                ct = 7;
            } else {
                put(c >> 19);
                c &= 0x7FFFF;
                ct = 8;
            }
        }
    }
    void renorm()
    {
        do {
            a <<= 1;
            c <<= 1;
            if (--ct == 0) byteout();
        } while ((a & 0x8000) == 0);
    }
    void encode(int d, int cx)
    {
        const int s = idx[cx];
        const uint32_t qe = kQe[s];
        a -= qe;
        if (d == mps[cx]) {
            if ((a & 0x8000) == 0) {
                if (a < qe) a = qe;
                else c += qe;
                idx[cx] = kNMPS[s];
                renorm();
            } else {
                c += qe;
            }
        } else {
            if (a < qe) c += qe;
            else a = qe;
            if (kSW[s]) mps[cx] ^= 1;
            idx[cx] = kNLPS[s];
            renorm();
        }
    }
    // FLUSH (ISO C.2.9) and return the codeword length.
    size_t flush()
    {
        const uint32_t tempc = c + a;
        c |= 0xFFFF;
        if (c >= tempc) c -= 0x8000;
        c <<= ct;
        byteout();
        c <<= ct;
        byteout();
        return buf[bp] == 0xFF ? bp - 1 : bp;
    }
};

// Raw (bypass) coding of ISO D.6: bits stored MSB first; a byte that
// follows 0xFF carries 7 bits (its MSB is a stuffed 0).  A segment that
// would end on 0xFF gets a zero byte, so it never ends on a marker prefix.
struct RawEnc {
    std::vector<uint8_t> buf;
    uint32_t cur = 0;
    int ct = 8;
    void restart()
    {
        buf.clear();
        cur = 0;
        ct = 8;
    }
    void put(uint32_t b)
    {
        cur = (cur << 1) | (b & 1u);
        if (--ct == 0) {
            buf.push_back((uint8_t)cur);
            ct = cur == 0xFF ? 7 : 8;
            cur = 0;
        }
    }
    size_t flush()
    {
        const int full = !buf.empty() && buf.back() == 0xFF ? 7 : 8;
        if (ct < full) buf.push_back((uint8_t)(cur << ct));
        if (!buf.empty() && buf.back() == 0xFF) buf.push_back(0);
        return buf.size();
    }
};

// Whether coding pass t (0: the first cleanup pass) ends a codeword
// segment under code-block style `style` (ISO D.4.2, D.6): every pass with
// TERMALL; with BYPASS the tenth pass, then each raw SPP+MRP pair and each
// cleanup pass after it.
inline bool pass_terminates(int style, int t)
{
    if (style & TC_CBLK_STYLE_TERMALL) return true;
    if (style & TC_CBLK_STYLE_BYPASS) return t == 9 || (t >= 10 && t % 3 != 1);
    return false;
}
// Whether pass t is raw-coded (BYPASS: SPP and MRP passes from the 11th on).
inline bool pass_raw(int style, int t) { return (style & TC_CBLK_STYLE_BYPASS) && t >= 10 && t % 3 != 0; }
// Codeword segments that passes [0, passes) span.
inline int pass_segments(int style, int passes)
{
    int n = passes > 0;
    for (int t = 0; t + 1 < passes; t++) n += pass_terminates(style, t);
    return n;
}

// ============================ Tier-1 encoder (ISO D) ========================

namespace {
struct T1Enc {
    int w, h, W;
    std::vector<uint8_t> sig, sgn, ref, vis;
    std::vector<uint32_t> mag;
    const int32_t *coef;
    int orient;
    int style = 0;     // code-block style (VSC read here)
    bool raw = false;  // the current pass is raw-coded (BYPASS)
    MQEnc mq;
    RawEnc rw;

    T1Enc(const int32_t *c, int w_, int h_, int o, int st)
        : w(w_), h(h_), W(w_ + 2), sig((w_ + 2) * (h_ + 2)), sgn(sig.size()), ref(sig.size()),
          vis(sig.size()), mag((size_t)w_ * h_), coef(c), orient(o), style(st)
    {
        for (int i = 0; i < w * h; i++) mag[i] = (uint32_t)std::abs((int64_t)coef[i]);
    }
    uint8_t &S(std::vector<uint8_t> &v, int x, int y) { return v[(y + 1) * W + x + 1]; }
    int bit(int x, int y, int p) const { return (mag[y * w + x] >> p) & 1; }
    int neg(int x, int y) const { return coef[y * w + x] < 0; }

    // Vertically causal contexts (VSC): the row below a stripe counts as
    // insignificant.
    bool below_hidden(int y) const { return (style & TC_CBLK_STYLE_VSC) && (y & 3) == 3; }
    void counts(int x, int y, int &hh, int &vv, int &dd)
    {
        const bool nb = !below_hidden(y);
        hh = S(sig, x - 1, y) + S(sig, x + 1, y);
        vv = S(sig, x, y - 1) + (nb ? S(sig, x, y + 1) : 0);
        dd = S(sig, x - 1, y - 1) + S(sig, x + 1, y - 1) + (nb ? S(sig, x - 1, y + 1) + S(sig, x + 1, y + 1) : 0);
    }
    void code(int d, int cx)
    {
        if (raw) rw.put((uint32_t)d);
        else mq.encode(d, cx);
    }
    int zc(int hh, int vv, int dd) const
    {
        if (orient == 1) std::swap(hh, vv);
        if (orient == 3) {
            const int hv = hh + vv;
            if (dd >= 3) return 8;
            if (dd == 2) return hv >= 1 ? 7 : 6;
            if (dd == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
            return hv >= 2 ? 2 : hv;
        }
        if (hh == 2) return 8;
        if (hh == 1) return vv >= 1 ? 7 : (dd >= 1 ? 6 : 5);
        if (vv == 2) return 4;
        if (vv == 1) return 3;
        return dd >= 2 ? 2 : dd;
    }
    void code_sign(int x, int y)
    {
        auto contrib = [&](int xx, int yy) { return S(sig, xx, yy) ? (S(sgn, xx, yy) ? -1 : 1) : 0; };
        int hc = contrib(x - 1, y) + contrib(x + 1, y);
        int vc = contrib(x, y - 1) + (below_hidden(y) ? 0 : contrib(x, y + 1));
        hc = std::max(-1, std::min(1, hc));
        vc = std::max(-1, std::min(1, vc));
        int cx, xr;
        if (hc == 0) {
            cx = vc == 0 ? 9 : 10;
            xr = vc < 0;
        } else {
            cx = 12 + hc * vc;
            xr = hc < 0;
        }
        const int s = neg(x, y);
        if (raw) rw.put((uint32_t)s);  // raw: the sign itself
        else mq.encode(s ^ xr, cx);
        S(sgn, x, y) = (uint8_t)s;
        S(sig, x, y) = 1;
    }
    void spp(int p)
    {
        for (int y0 = 0; y0 < h; y0 += 4)
            for (int x = 0; x < w; x++)
                for (int y = y0; y < std::min(h, y0 + 4); y++) {
                    int hh, vv, dd;
                    if (S(sig, x, y)) continue;
                    counts(x, y, hh, vv, dd);
                    if (hh + vv + dd == 0) continue;
                    S(vis, x, y) = 1;
                    const int b = bit(x, y, p);
                    code(b, zc(hh, vv, dd));
                    if (b) code_sign(x, y);
                }
    }
    void mrp(int p)
    {
        for (int y0 = 0; y0 < h; y0 += 4)
            for (int x = 0; x < w; x++)
                for (int y = y0; y < std::min(h, y0 + 4); y++) {
                    int hh, vv, dd;
                    if (!S(sig, x, y) || S(vis, x, y)) continue;
                    counts(x, y, hh, vv, dd);
                    code(bit(x, y, p), S(ref, x, y) ? 16 : (hh + vv + dd ? 15 : 14));
                    S(ref, x, y) = 1;
                }
    }
    void cup(int p)
    {
        for (int y0 = 0; y0 < h; y0 += 4)
            for (int x = 0; x < w; x++) {
                int y = y0;
                if (y0 + 4 <= h) {
                    bool ok = true;
                    for (int k = 0; k < 4 && ok; k++) {
                        int hh, vv, dd;
                        if (S(sig, x, y0 + k) || S(vis, x, y0 + k)) { ok = false; break; }
                        counts(x, y0 + k, hh, vv, dd);
                        if (hh + vv + dd) ok = false;
                    }
                    if (ok) {
                        int r = -1;
                        for (int k = 0; k < 4; k++)
                            if (bit(x, y0 + k, p)) { r = k; break; }
                        if (r < 0) {
                            mq.encode(0, 18);
                            continue;
                        }
                        mq.encode(1, 18);
                        mq.encode(r >> 1, 17);
                        mq.encode(r & 1, 17);
                        code_sign(x, y0 + r);
                        y = y0 + r + 1;
                    }
                }
                for (; y < std::min(h, y0 + 4); y++) {
                    int hh, vv, dd;
                    if (S(sig, x, y) || S(vis, x, y)) continue;
                    counts(x, y, hh, vv, dd);
                    const int b = bit(x, y, p);
                    mq.encode(b, zc(hh, vv, dd));
                    if (b) code_sign(x, y);
                }
            }
    }
};
}  // namespace

int t1_encode_block(const int32_t *coef, int w, int h, int orient, int mb, int passes,
                    std::vector<uint8_t> &out, int *passes_out, int *zero_bitplanes, int style,
                    std::vector<std::pair<uint32_t, int>> *segments)
{
    if (segments) segments->clear();
    if (w < 1 || h < 1 || w > 64 || h > 64 || orient < 0 || orient > 3 || mb < 1 || mb > 31)
        return TC_E_ARG;
    uint32_t mx = 0;
    for (int i = 0; i < w * h; i++) mx = std::max(mx, (uint32_t)std::abs((int64_t)coef[i]));
    int numbps = 0;
    while (numbps < 32 && (mx >> numbps)) numbps++;
    if (numbps > mb) return TC_E_ARG;
    *zero_bitplanes = mb - numbps;
    out.clear();
    if (numbps == 0) {
        *passes_out = 0;
        return TC_OK;
    }
    const int total = 3 * numbps - 2;
    if (passes <= 0 || passes > total) passes = total;
    T1Enc e(coef, w, h, orient, style);
    out.clear();
    int done = 0, seg_passes = 0;
    // ends the current codeword segment (MQ FLUSH or raw padding)
    auto terminate = [&]() {
        size_t len;
        if (e.raw) {
            len = e.rw.flush();
            out.insert(out.end(), e.rw.buf.begin(), e.rw.buf.end());
            e.rw.restart();
        } else {
            len = e.mq.flush();
            out.insert(out.end(), e.mq.buf.begin() + 1, e.mq.buf.begin() + 1 + len);
            e.mq.restart();
        }
        if (segments) segments->emplace_back((uint32_t)len, seg_passes);
        seg_passes = 0;
    };
    // after pass t: context reset, termination
    auto pass_done = [&](int t) {
        if (style & TC_CBLK_STYLE_RESET) e.mq.reset_contexts();
        ++seg_passes;
        if (t + 1 == passes || pass_terminates(style, t)) terminate();
    };
    for (int p = numbps - 1; p >= 0 && done < passes; p--) {
        if (p != numbps - 1) {
            e.raw = pass_raw(style, done);
            e.spp(p);
            pass_done(done);
            if (++done >= passes) break;
            e.raw = pass_raw(style, done);
            e.mrp(p);
            pass_done(done);
            if (++done >= passes) break;
        }
        e.raw = false;
        e.cup(p);
        if (style & TC_CBLK_STYLE_SEGSYM)  // segmentation symbol 1010 (ISO D.5)
            for (int b : {1, 0, 1, 0}) e.mq.encode(b, 17);
        pass_done(done);
        ++done;
        std::fill(e.vis.begin(), e.vis.end(), 0);
    }
    *passes_out = passes;
    return TC_OK;
}

// ============================ bit I/O and tag trees =========================

namespace {
struct BitWriter {
    std::vector<uint8_t> &out;
    uint32_t cur = 0;
    int ct = 8;
    explicit BitWriter(std::vector<uint8_t> &o) : out(o) {}
    void put(int b)
    {
        if (ct == 0) {
            out.push_back((uint8_t)cur);
            ct = (cur == 0xFF) ? 7 : 8;
            cur = 0;
        }
        ct--;
        cur |= (uint32_t)(b & 1) << ct;
    }
    void put_bits(uint32_t v, int n)
    {
        for (int i = n - 1; i >= 0; i--) put((v >> i) & 1);
    }
    // Packet header end (ISO B.10.1): emit the partial byte; a final 0xFF is
    // followed by a zero byte so the header never ends on 0xFF.
    void flush()
    {
        out.push_back((uint8_t)cur);
        if (cur == 0xFF) out.push_back(0);
        cur = 0;
        ct = 8;
    }
};

struct BitReader {
    const uint8_t *p;
    size_t pos, end;
    uint32_t cur = 0;
    int ct = 0;
    bool overrun = false;
    BitReader(const uint8_t *d, size_t start, size_t e) : p(d), pos(start), end(e) {}
    int get()
    {
        if (ct == 0) {
            const bool ff = (cur == 0xFF);
            if (pos >= end) {
                overrun = true;
                cur = 0;
            } else {
                cur = p[pos++];
            }
            ct = ff ? 7 : 8;
        }
        ct--;
        return (cur >> ct) & 1;
    }
    uint32_t get_bits(int n)
    {
        uint32_t v = 0;
        for (int i = 0; i < n; i++) v = (v << 1) | (uint32_t)get();
        return v;
    }
    void align()
    {
        if (cur == 0xFF) {
            if (pos >= end) overrun = true;
            else pos++;
        }
        cur = 0;
        ct = 0;
    }
};

// Tag tree (ISO B.10.2) over a gw x gh grid of leaves.
struct TagTree {
    struct Node {
        int parent;
        int value;
        int low;
        bool known;
    };
    std::vector<Node> nodes;
    int gw = 0, gh = 0;
    TagTree(int w, int h) : gw(w), gh(h)
    {
        std::vector<std::pair<int, int>> dims;
        int cw = w, ch = h;
        do {
            dims.emplace_back(cw, ch);
            cw = (cw + 1) / 2;
            ch = (ch + 1) / 2;
        } while (dims.back().first * dims.back().second > 1);
        int total = 0;
        for (auto &d : dims) total += d.first * d.second;
        nodes.assign(total, Node{-1, 0x7FFFFFFF, 0, false});
        int off = 0;
        for (size_t l = 0; l + 1 < dims.size(); l++) {
            const int lw = dims[l].first, lh = dims[l].second;
            const int poff = off + lw * lh;
            const int pw = dims[l + 1].first;
            for (int y = 0; y < lh; y++)
                for (int x = 0; x < lw; x++) nodes[off + y * lw + x].parent = poff + (y / 2) * pw + x / 2;
            off = poff;
        }
    }
    void set_leaves(const std::vector<int> &vals)
    {
        for (auto &n : nodes) n.value = 0x7FFFFFFF;
        for (size_t i = 0; i < vals.size(); i++) {
            int k = (int)i;
            while (k >= 0) {
                nodes[k].value = std::min(nodes[k].value, vals[i]);
                k = nodes[k].parent;
            }
        }
    }
    void path(int leaf, int *stk, int &n) const
    {
        n = 0;
        for (int k = leaf; k >= 0; k = nodes[k].parent) stk[n++] = k;
    }
    void encode(BitWriter &bw, int leaf, int threshold)
    {
        int stk[40], n;
        path(leaf, stk, n);
        int low = 0;
        for (int i = n - 1; i >= 0; i--) {
            Node &nd = nodes[stk[i]];
            if (low > nd.low) nd.low = low;
            else low = nd.low;
            while (low < threshold) {
                if (low >= nd.value) {
                    if (!nd.known) {
                        bw.put(1);
                        nd.known = true;
                    }
                    break;
                }
                bw.put(0);
                low++;
            }
            nd.low = low;
        }
    }
    // Returns 1 when the leaf's value is below threshold.
    int decode(BitReader &br, int leaf, int threshold)
    {
        int stk[40], n;
        path(leaf, stk, n);
        int low = 0;
        for (int i = n - 1; i >= 0; i--) {
            Node &nd = nodes[stk[i]];
            if (low > nd.low) nd.low = low;
            else low = nd.low;
            while (low < threshold && low < nd.value) {
                if (br.get()) nd.value = low;
                else low++;
                if (br.overrun) return 0;
            }
            nd.low = low;
        }
        return nodes[leaf].value < threshold;
    }
    // Decodes the leaf's value outright (one walk from the root instead of
    // one per threshold); -1 when the bits run out or the value passes limit.
    int decode_value(BitReader &br, int leaf, int limit)
    {
        int stk[40], n;
        path(leaf, stk, n);
        int low = 0;
        for (int i = n - 1; i >= 0; i--) {
            Node &nd = nodes[stk[i]];
            if (low > nd.low) nd.low = low;
            else low = nd.low;
            while (low < nd.value) {
                if (low > limit) return -1;
                if (br.get()) nd.value = low;
                else low++;
                if (br.overrun) return -1;
            }
            nd.low = low;
        }
        return nodes[leaf].value;
    }
    void reset_decoder()
    {
        for (auto &n : nodes) {
            n.value = 0x7FFFFFFF;
            n.low = 0;
            n.known = false;
        }
    }
};

static void put_num_passes(BitWriter &bw, int n)
{
    if (n == 1) bw.put(0);
    else if (n == 2) bw.put_bits(2, 2);
    else if (n <= 5) { bw.put_bits(3, 2); bw.put_bits(n - 3, 2); }
    else if (n <= 36) { bw.put_bits(0xF, 4); bw.put_bits(n - 6, 5); }
    else { bw.put_bits(0x1FF, 9); bw.put_bits(n - 37, 7); }
}

// ISO Table B.4 (decode_num_coding_passes, codestream.c:300-313).
static int get_num_passes(BitReader &br)
{
    if (!br.get()) return 1;
    if (!br.get()) return 2;
    int n = (int)br.get_bits(2);
    if (n != 3) return 3 + n;
    n = (int)br.get_bits(5);
    if (n != 31) return 6 + n;
    return 37 + (int)br.get_bits(7);
}

static int floorlog2(int a)
{
    int l = 0;
    while (a > 1) { a >>= 1; l++; }
    return l;
}
}  // namespace

// ============================ codestream markers ============================

enum : uint16_t {
    M_SOC = 0xFF4F, M_SIZ = 0xFF51, M_COD = 0xFF52, M_COC = 0xFF53, M_TLM = 0xFF55,
    M_PLM = 0xFF57, M_PLT = 0xFF58, M_QCD = 0xFF5C, M_QCC = 0xFF5D, M_RGN = 0xFF5E,
    M_POC = 0xFF5F, M_PPM = 0xFF60, M_PPT = 0xFF61, M_CRG = 0xFF63, M_COM = 0xFF64,
    M_SOT = 0xFF90, M_SOP = 0xFF91, M_EPH = 0xFF92, M_SOD = 0xFF93, M_EOC = 0xFFD9
};

namespace {
struct Writer {
    std::vector<uint8_t> &o;
    void u8(uint32_t v) { o.push_back((uint8_t)v); }
    void u16(uint32_t v) { u8(v >> 8); u8(v); }
    void u32(uint32_t v) { u16(v >> 16); u16(v & 0xFFFF); }
};

struct Reader {
    const uint8_t *d;
    size_t len, pos = 0;
    bool bad = false;
    uint32_t u8()
    {
        if (pos + 1 > len) { bad = true; return 0; }
        return d[pos++];
    }
    uint32_t u16() { uint32_t a = u8(); return (a << 8) | u8(); }
    uint32_t u32() { uint32_t a = u16(); return (a << 16) | u16(); }
};

// Coding style of a component: SPcod of COD, SPcoc of COC (ISO A.6.1-A.6.2).
struct Coding {
    int levels = 0, xcb = 6, ycb = 6, cblk_style = 0, reversible = 1;
    std::vector<int> ppx, ppy;  // precinct size exponents per resolution
};

// Quantisation of a component: QCD or QCC (ISO A.6.4-A.6.5).
struct Quant {
    int qstyle = 0, guard = 2;
    std::vector<int> eps, mu;  // as signalled (1 or 3N+1 entries)
};

// One progression volume of a POC marker (ISO A.6.6): layers [0, lye),
// resolutions [rs, re), components [cs, ce) in order prog.
struct PocEntry {
    int rs, cs, lye, re, ce, prog;
};

// The coding parameters one header sets: the main header, or a tile's
// tile-part headers (COD / COC / QCD / QCC in the first one, POC in any).
// Per component, a COC / QCC replaces the header's COD / QCD.
struct Scope {
    std::vector<PocEntry> poc;
    bool has_cod = false, has_qcd = false;
    int scod = 0, prog = 0, layers = 1, mct = 0;
    Coding cod;
    Quant qcd;
    std::vector<char> has_coc, has_qcc;
    std::vector<Coding> coc;
    std::vector<Quant> qcc;
    std::vector<char> has_roi;  // RGN (ISO A.6.3): maxshift value per component
    std::vector<int> roi;
    void init(int ncomp)
    {
        has_coc.assign(ncomp, 0);
        has_qcc.assign(ncomp, 0);
        coc.resize(ncomp);
        qcc.resize(ncomp);
        has_roi.assign(ncomp, 0);
        roi.assign(ncomp, 0);
    }
};

struct Params {
    int width = 0, height = 0, ncomp = 0, bits = 0, is_signed = 0;
    // reference grid (ISO B.2): image [xo, xs) x [yo, ys); tiles of tw x th
    // anchored at (xto, yto)
    int64_t xs = 0, ys = 0, xo = 0, yo = 0, xto = 0, yto = 0;
    int tw = 0, th = 0;
    int dx[4] = {1, 1, 1, 1}, dy[4] = {1, 1, 1, 1};  // component subsampling XRsiz, YRsiz
    bool subsampled = false;
    Scope main;
    int levels = 0;  // decomposition levels, shared by every component and tile
    bool have_siz = false;
    // tiles in raster order, on the reference grid: [x0, x1) x [y0, y1)
    struct Tile {
        int64_t x0, y0, x1, y1;
    };
    std::vector<Tile> tiles;
    // packed packet headers of the main header (PPM, ISO A.7.4): Zppm and
    // the segment's Ippm bytes
    std::vector<std::pair<int, std::vector<uint8_t>>> ppm;
};

// Precedence of ISO A.6: tile COC > tile COD > main COC > main COD, and
// likewise for QCC / QCD.  t: the tile's header scope, or null.
const Coding &coding_of(const Params &P, const Scope *t, int c)
{
    if (t && t->has_coc[c]) return t->coc[c];
    if (t && t->has_cod) return t->cod;
    if (P.main.has_coc[c]) return P.main.coc[c];
    return P.main.cod;
}

const Quant &quant_of(const Params &P, const Scope *t, int c)
{
    if (t && t->has_qcc[c]) return t->qcc[c];
    if (t && t->has_qcd) return t->qcd;
    if (P.main.has_qcc[c]) return P.main.qcc[c];
    return P.main.qcd;
}

// ROI maxshift of component c: a tile's RGN, else the main header's, else 0.
int roi_of(const Params &P, const Scope *t, int c)
{
    if (t && t->has_roi[c]) return t->roi[c];
    return P.main.has_roi[c] ? P.main.roi[c] : 0;
}

// Progression, layers, SOP/EPH and the colour transform come from COD only.
const Scope &cod_scope(const Params &P, const Scope *t) { return t && t->has_cod ? *t : P.main; }
}  // namespace

// SPcod / SPcoc: levels, code-block size and style, wavelet, precincts.
static int read_spcod(Reader &rd, bool precincts, Coding &c, std::string &err)
{
    c.levels = (int)rd.u8();
    c.xcb = (int)rd.u8() + 2;
    c.ycb = (int)rd.u8() + 2;
    c.cblk_style = (int)rd.u8();
    c.reversible = (int)rd.u8();
    if (c.levels > 32 || c.xcb > 10 || c.ycb > 10 || c.xcb + c.ycb > 12) { err = "bad COD/COC"; return TC_E_CODESTREAM; }
    if (c.xcb > 6 || c.ycb > 6) { err = "code-blocks larger than 64x64"; return TC_E_UNSUPPORTED; }
    if (c.cblk_style & ~0x3F) { err = "unknown code-block style bits"; return TC_E_UNSUPPORTED; }
    if (c.reversible > 1) { err = "unknown wavelet"; return TC_E_CODESTREAM; }
    c.ppx.assign(c.levels + 1, 15);
    c.ppy.assign(c.levels + 1, 15);
    if (precincts)
        for (int r = 0; r <= c.levels; r++) {
            const uint32_t v = rd.u8();
            c.ppx[r] = (int)(v & 0xF);
            c.ppy[r] = (int)(v >> 4);
        }
    return TC_OK;
}

// Sqcd / Sqcc and the step sizes up to the end of the marker segment.
static int read_quant(Reader &rd, size_t seg_end, Quant &q, std::string &err)
{
    const uint32_t s = rd.u8();
    q.qstyle = (int)(s & 0x1F);
    q.guard = (int)(s >> 5);
    q.eps.clear();
    q.mu.clear();
    if (q.qstyle == 0) {
        while (rd.pos < seg_end) q.eps.push_back((int)(rd.u8() >> 3)), q.mu.push_back(0);
    } else if (q.qstyle == 1 || q.qstyle == 2) {
        while (rd.pos + 1 < seg_end) {
            const uint32_t v = rd.u16();
            q.eps.push_back((int)(v >> 11));
            q.mu.push_back((int)(v & 0x7FF));
        }
    } else {
        err = "bad quantisation style";
        return TC_E_CODESTREAM;
    }
    return TC_OK;
}

// COD, COC, QCD and QCC of a main or tile-part header into scope S.  The
// reference's parser reads COD and QCD (read_cod_marker, read_qcd_marker,
// codestream.c:95-230) and leaves COC/QCC as a stub (codestream.c:137-140).
static int read_coding_marker(Reader &rd, uint32_t m, size_t seg_end, int ncomp, Scope &S, std::string &err)
{
    int rc;
    if (m == M_COD) {
        S.scod = (int)rd.u8();
        S.prog = (int)rd.u8();
        S.layers = (int)rd.u16();
        S.mct = (int)rd.u8();
        if (S.prog > 4 || S.layers < 1) { err = "bad progression or layer count"; return TC_E_CODESTREAM; }
        if ((rc = read_spcod(rd, S.scod & 1, S.cod, err))) return rc;
        S.has_cod = true;
    } else if (m == M_QCD) {
        if ((rc = read_quant(rd, seg_end, S.qcd, err))) return rc;
        S.has_qcd = true;
    } else {
        const int c = (int)(ncomp < 257 ? rd.u8() : rd.u16());
        if (c >= ncomp) { err = "COC/QCC for a component that does not exist"; return TC_E_CODESTREAM; }
        if (m == M_COC) {
            const int scoc = (int)rd.u8();
            if ((rc = read_spcod(rd, scoc & 1, S.coc[c], err))) return rc;
            S.has_coc[c] = 1;
        } else {
            if ((rc = read_quant(rd, seg_end, S.qcc[c], err))) return rc;
            S.has_qcc[c] = 1;
        }
    }
    if (rd.bad || rd.pos > seg_end) { err = "truncated coding marker"; return TC_E_CODESTREAM; }
    return TC_OK;
}

// POC (ISO A.6.6): progression volumes appended to `poc`.  The reference
// reads one progression order from COD (codestream.c:95-136).
// RGN (ISO A.6.3): Crgn, Srgn (0: the maxshift method of Annex H), SPrgn.
static int read_rgn(Reader &rd, size_t seg_end, int ncomp, Scope &S, std::string &err)
{
    const int c = ncomp < 257 ? (int)rd.u8() : (int)rd.u16();
    const int style = (int)rd.u8(), shift = (int)rd.u8();
    if (rd.bad || rd.pos > seg_end || c >= ncomp) { err = "bad RGN"; return TC_E_CODESTREAM; }
    if (style != 0) { err = "RGN styles other than maxshift"; return TC_E_UNSUPPORTED; }
    S.has_roi[c] = 1;
    S.roi[c] = shift;
    return TC_OK;
}

static int read_poc(Reader &rd, size_t seg_end, int ncomp, std::vector<PocEntry> &poc, std::string &err)
{
    const bool wide = ncomp >= 257;
    const size_t entry = wide ? 9 : 7;
    while (rd.pos + entry <= seg_end) {
        PocEntry e;
        e.rs = (int)rd.u8();
        e.cs = (int)(wide ? rd.u16() : rd.u8());
        e.lye = (int)rd.u16();
        e.re = (int)rd.u8();
        e.ce = (int)(wide ? rd.u16() : rd.u8());
        if (!wide && e.ce == 0) e.ce = 256;
        e.prog = (int)rd.u8();
        if (e.prog > 4 || e.re <= e.rs || e.ce <= e.cs) { err = "bad POC entry"; return TC_E_CODESTREAM; }
        poc.push_back(e);
    }
    if (rd.bad || rd.pos != seg_end) { err = "bad POC length"; return TC_E_CODESTREAM; }
    return TC_OK;
}

// Every component of the image (t null) or of a tile must share the
// decomposition levels and the wavelet, and every tile the colour transform:
// the DWT launches and the fused colour stage need one geometry per image.
static int check_coding(const Params &P, const Scope *t, std::string &err)
{
    const Coding &c0 = P.main.cod;
    for (int c = 0; c < P.ncomp; c++) {
        const Coding &k = coding_of(P, t, c);
        if (k.levels != c0.levels || k.reversible != c0.reversible) {
            err = "components or tiles with different decomposition levels or wavelets are not supported";
            return TC_E_UNSUPPORTED;
        }
    }
    if (cod_scope(P, t).mct != P.main.mct) {
        err = "tiles with different colour transforms are not supported";
        return TC_E_UNSUPPORTED;
    }
    return TC_OK;
}

// Tile grid (ISO B.3): tile (p, q) covers [max(XTOsiz + p*XTsiz, XOsiz),
// min(XTOsiz + (p+1)*XTsiz, Xsiz)) horizontally, likewise vertically, as
// the reference's init_tiles places tile p, q at p*tile_w, q*tile_h
// (codestream_image.c:256-270) for a grid without offsets.  Each tile's
// origin must be a multiple of 2^levels: the tile's subbands, and so its
// reverse DWT, then have the geometry of an image of the tile's size at the
// origin.
static int tile_grid(Params &P, std::string &err)
{
    const int64_t nx = (P.xs - P.xto + P.tw - 1) / P.tw, ny = (P.ys - P.yto + P.th - 1) / P.th;
    if (nx * ny > 65535) { err = "more than 65535 tiles"; return TC_E_CODESTREAM; }
    const int64_t mask = (P.levels >= 62 ? INT64_MAX : ((int64_t)1 << P.levels) - 1);
    P.tiles.clear();
    for (int64_t q = 0; q < ny; q++)
        for (int64_t p = 0; p < nx; p++) {
            Params::Tile t;
            t.x0 = std::max(P.xto + p * P.tw, P.xo);
            t.y0 = std::max(P.yto + q * P.th, P.yo);
            t.x1 = std::min(P.xto + (p + 1) * P.tw, P.xs);
            t.y1 = std::min(P.yto + (q + 1) * P.th, P.ys);
            if ((t.x0 & mask) || (t.y0 & mask)) {
                err = "tile or image origins that are not multiples of 2^levels are not supported";
                return TC_E_UNSUPPORTED;
            }
            P.tiles.push_back(t);
        }
    return TC_OK;
}

static int parse_main(Reader &rd, Params &P, std::string &err)
{
    if (rd.u16() != M_SOC) { err = "missing SOC marker"; return TC_E_CODESTREAM; }
    for (;;) {
        const uint32_t m = rd.u16();
        if (rd.bad) { err = "truncated main header"; return TC_E_CODESTREAM; }
        if (m == M_SOT) { rd.pos -= 2; break; }
        if ((m >> 8) != 0xFF) { err = "expected a marker in the main header"; return TC_E_CODESTREAM; }
        const uint32_t L = rd.u16();
        const size_t seg_end = rd.pos - 2 + L;
        if (L < 2 || seg_end > rd.len) { err = "bad marker segment length"; return TC_E_CODESTREAM; }
        switch (m) {
        case M_SIZ: {
            rd.u16();  // Rsiz
            const uint32_t xs = rd.u32(), ys = rd.u32(), xo = rd.u32(), yo = rd.u32();
            const uint32_t xt = rd.u32(), yt = rd.u32(), xto = rd.u32(), yto = rd.u32();
            const uint32_t c = rd.u16();
            if (xo >= xs || yo >= ys || xt == 0 || yt == 0 || xto > xo || yto > yo ||
                (uint64_t)xto + xt <= xo || (uint64_t)yto + yt <= yo) {
                err = "bad image or tile geometry in SIZ";
                return TC_E_CODESTREAM;
            }
            if (c < 1 || c > 4) { err = "1 to 4 components supported"; return TC_E_UNSUPPORTED; }
            if (xs - xo > 65535 || ys - yo > 65535) { err = "image size out of range"; return TC_E_UNSUPPORTED; }
            P.xs = xs; P.ys = ys; P.xo = xo; P.yo = yo; P.xto = xto; P.yto = yto;
            P.width = (int)(xs - xo); P.height = (int)(ys - yo);
            P.tw = (int)std::min<uint32_t>(xt, 0x7FFFFFFF);
            P.th = (int)std::min<uint32_t>(yt, 0x7FFFFFFF);
            P.ncomp = (int)c;
            for (uint32_t i = 0; i < c; i++) {
                const uint32_t ss = rd.u8(), dx = rd.u8(), dy = rd.u8();
                const int b = (int)(ss & 0x7F) + 1, sg = (int)(ss >> 7);
                if (dx < 1 || dy < 1) { err = "bad component subsampling"; return TC_E_CODESTREAM; }
                if (i < 4) {
                    P.dx[i] = (int)dx;
                    P.dy[i] = (int)dy;
                }
                if (dx != 1 || dy != 1) P.subsampled = true;
                if (i == 0) { P.bits = b; P.is_signed = sg; }
                else if (b != P.bits || sg != P.is_signed) { err = "components must share bit depth"; return TC_E_UNSUPPORTED; }
            }
            if (P.bits > 16) { err = "bit depth above 16"; return TC_E_UNSUPPORTED; }
            P.main.init(P.ncomp);
            P.have_siz = true;
            break;
        }
        case M_COD: case M_COC: case M_QCD: case M_QCC: {
            if (!P.have_siz) { err = "coding marker before SIZ"; return TC_E_CODESTREAM; }
            const int rc = read_coding_marker(rd, m, seg_end, P.ncomp, P.main, err);
            if (rc) return rc;
            break;
        }
        case M_POC: {
            if (!P.have_siz) { err = "POC before SIZ"; return TC_E_CODESTREAM; }
            const int rc = read_poc(rd, seg_end, P.ncomp, P.main.poc, err);
            if (rc) return rc;
            break;
        }
        case M_PPM: {
            if (seg_end - rd.pos < 1) { err = "bad PPM"; return TC_E_CODESTREAM; }
            const int z = (int)rd.u8();
            P.ppm.emplace_back(z, std::vector<uint8_t>(rd.d + rd.pos, rd.d + seg_end));
            break;
        }
        case M_RGN: {
            if (!P.have_siz) { err = "RGN before SIZ"; return TC_E_CODESTREAM; }
            const int rc = read_rgn(rd, seg_end, P.ncomp, P.main, err);
            if (rc) return rc;
            break;
        }
        default:
            break;  // COM, TLM, PLM, CRG (display registration) and others change no sample
        }
        rd.pos = seg_end;
    }
    if (!P.have_siz || !P.main.has_cod || !P.main.has_qcd) {
        err = "main header lacks SIZ, COD or QCD";
        return TC_E_CODESTREAM;
    }
    P.levels = P.main.cod.levels;
    int rc = check_coding(P, nullptr, err);
    if (rc) return rc;
    if ((rc = tile_grid(P, err))) return rc;
    if (P.subsampled) {
        // subsampled components: one tile at the origin; the colour
        // transform only over components 0-2 of one size
        if (P.tiles.size() != 1 || P.xo || P.yo) {
            err = "subsampled components in tiled or offset images are not supported";
            return TC_E_UNSUPPORTED;
        }
        if (P.main.mct && P.ncomp >= 3 &&
            (P.dx[1] != P.dx[0] || P.dx[2] != P.dx[0] || P.dy[1] != P.dy[0] || P.dy[2] != P.dy[0])) {
            err = "a colour transform over components of different sizes";
            return TC_E_CODESTREAM;
        }
    }
    return TC_OK;
}

// Image information from the main header (COD and QCD; per-component COC /
// QCC values and tile-part headers may differ in code-block size and
// quantisation).
static void fill_info(const Params &P, tc_image_info &info)
{
    std::memset(&info, 0, sizeof info);
    info.width = P.width;
    info.height = P.height;
    info.ncomp = P.ncomp;
    info.bits = P.bits;
    info.is_signed = P.is_signed;
    info.levels = P.levels;
    info.reversible = P.main.cod.reversible;
    info.mct = P.main.mct;
    info.cblk_w = 1 << P.main.cod.xcb;
    info.cblk_h = 1 << P.main.cod.ycb;
    info.layers = P.main.layers;
    info.progression = P.main.prog;
    info.guard_bits = P.main.qcd.guard;
    info.quant_style = P.main.qcd.qstyle;
    info.ntiles = (uint32_t)P.tiles.size();
    for (int c = 0; c < 4; c++) {
        info.comp_dx[c] = (uint8_t)(c < P.ncomp ? P.dx[c] : 1);
        info.comp_dy[c] = (uint8_t)(c < P.ncomp ? P.dy[c] : 1);
    }
}

static int read_raw_header(const uint8_t *cs, size_t len, tc_image_info &info, std::string &err)
{
    Reader rd{cs, len};
    Params P;
    const int rc = parse_main(rd, P, err);
    if (rc) return rc;
    fill_info(P, info);
    return TC_OK;
}

// Quantisation parameters per band (ISO A.6.4-A.6.5, E.1).  Derived style
// restates read_qcd_marker (codestream.c:142-230) with ISO's exponent rule.
static int assign_quant(const Quant &Q, int bits, int levels, std::vector<Resolution> &res, std::string &err)
{
    int bi = 0;
    for (int r = 0; r <= levels; r++)
        for (Band &b : res[r].bands) {
            int eps, mu;
            if (Q.qstyle == 1) {
                if (Q.eps.empty()) { err = "empty QCD/QCC"; return TC_E_CODESTREAM; }
                eps = Q.eps[0] - levels + b.level;
                mu = Q.mu[0];
                if (eps < 0) eps = 0;
            } else {
                if (bi >= (int)Q.eps.size()) { err = "QCD/QCC has too few subbands"; return TC_E_CODESTREAM; }
                eps = Q.eps[bi];
                mu = Q.mu[bi];
            }
            bi++;
            b.eps = eps;
            b.mu = mu;
            b.mb = Q.guard + eps - 1;
            if (b.mb > 31) { err = "more than 31 magnitude bit-planes"; return TC_E_UNSUPPORTED; }
            const int rb = bits + band_gain_log2(b.orient);
            b.step = (float)std::ldexp(1.0 + mu / 2048.0, rb - eps);
        }
    return TC_OK;
}

namespace {
// A code-block's codeword segments (one per layer that adds bytes) are a
// list threaded through the tile's segment arena.
struct SegNode {
    size_t off;    // in the codestream
    uint32_t len;
    int next;
};

struct CblkState {
    int included = 0;
    int lblock = 3;
    int zbp = 0;
    int passes = 0;
    int head = -1, tail = -1, nseg = 0;  // segment list in the tile's arena
    uint64_t bytes = 0;
    std::vector<uint32_t> seglen;  // BYPASS / TERMALL: codeword segment lengths
};

// Descriptors of all tiles before their segments are placed: each entry's
// segments are segs[first[k] .. first[k+1]).
struct Emit {
    std::vector<std::pair<size_t, uint32_t>> segs;
    std::vector<uint32_t> first;
    bool multi = false;  // some block has more than one segment
    // Blocks whose codeword segments are terminated (BYPASS / TERMALL):
    // descriptor index and its segment lengths at tab[at .. at + n).
    struct Table {
        size_t desc;
        uint32_t at, n;
    };
    std::vector<Table> tables;
    std::vector<uint32_t> tab;
};
}  // namespace

// Packets of one tile (ISO B.9-B.10) read from its tile-parts `parts` (packet
// data ranges in codestream order), and its code-block descriptors appended
// to out.desc with coefficients at element coef_off of the image's arena.
// Follows decode_tiles / decode_packet_header / decode_packet_body
// (codestream.c:336-510), one call per tile as decode_codestream loops over
// the tiles (codestream.c:524-527).
static int parse_tile(const uint8_t *cs, size_t len, const Params &P, const Params::Tile &T, const Scope &ts,
                      const std::vector<std::pair<size_t, size_t>> &parts, uint64_t coef_off, Parsed &out,
                      Emit &em, std::string &err, const std::vector<uint8_t> *packed = nullptr)
{
    int rc;
    if ((rc = check_coding(P, &ts, err))) return rc;
    const Scope &cs_ = cod_scope(P, &ts);
    const int NL = P.levels, R = NL + 1, C = P.ncomp, L = cs_.layers, scod = cs_.scod, prog = cs_.prog;
    const bool reversible = P.main.cod.reversible != 0;

    // Precinct partition of each resolution (ISO B.6): 2^PPx x 2^PPy cells
    // of the resolution's grid; in a subband of resolution r > 0 the cells
    // are 2^(PPx-1) x 2^(PPy-1), and code-blocks are capped to fit them (B.7).
    struct PrecBand {
        int i0 = 0, i1 = 0, j0 = 0, j1 = 0;  // the band's code-blocks inside the precinct
        TagTree incl{1, 1}, zbp{1, 1};
    };
    struct ResState {
        int64_t rx0 = 0, ry0 = 0;  // the resolution's origin on its own grid
        int px = 15, py = 15;      // precinct size exponents
        int pw = 0, ph = 0;        // precincts across and down
        std::vector<std::vector<CblkState>> cb;   // per band: its code-blocks
        std::vector<std::vector<PrecBand>> prec;  // per precinct: per band
    };
    // Per component (its own code-block and precinct sizes and quantisation,
    // COC / QCC): subband geometry, then per resolution the code-block
    // states of each band and per precinct each band's block range and tag
    // trees.  With the tile origin a multiple of 2^levels the subband sizes
    // are those of a tw x th image at the origin; the code-block and
    // precinct grids, anchored at the reference grid's origin, depend on
    // where the tile is.
    std::vector<std::vector<Resolution>> geo(C);
    std::vector<std::vector<ResState>> st(C, std::vector<ResState>(R));
    std::vector<int> style(C);  // code-block style per component (COD / COC)
    for (int c = 0; c < C; c++) style[c] = coding_of(P, &ts, c).cblk_style;
    // the tile on each component's grid (ISO B.3: ceil of the reference-grid
    // box over the subsampling), its plane size and offset in the arena
    std::vector<Params::Tile> tc(C);
    std::vector<uint64_t> coff(C + 1, 0);
    for (int c = 0; c < C; c++) {
        const int64_t dx = c < 4 ? P.dx[c] : 1, dy = c < 4 ? P.dy[c] : 1;
        tc[c] = Params::Tile{(T.x0 + dx - 1) / dx, (T.y0 + dy - 1) / dy, (T.x1 + dx - 1) / dx, (T.y1 + dy - 1) / dy};
        coff[c + 1] = coff[c] + (uint64_t)(tc[c].x1 - tc[c].x0) * (tc[c].y1 - tc[c].y0);
    }
    int64_t nprec_bands = 0;
    for (int c = 0; c < C; c++) {
        const Coding &cd = coding_of(P, &ts, c);
        const Params::Tile &Tc = tc[c];
        geo[c] = make_geometry((int)(Tc.x1 - Tc.x0), (int)(Tc.y1 - Tc.y0), NL, cd.xcb, cd.ycb);
        for (int r = 0; r <= NL; r++) {
            const int px = cd.ppx[r], py = cd.ppy[r];
            const int xcb = std::min(cd.xcb, r ? px - 1 : px), ycb = std::min(cd.ycb, r ? py - 1 : py);
            if (xcb < 0 || ycb < 0) { err = "bad precinct size"; return TC_E_CODESTREAM; }
            const int sh = NL - r;
            ResState &rs = st[c][r];
            const int64_t rx1 = (Tc.x1 + ((int64_t)1 << sh) - 1) >> sh, ry1 = (Tc.y1 + ((int64_t)1 << sh) - 1) >> sh;
            rs.rx0 = (Tc.x0 + ((int64_t)1 << sh) - 1) >> sh;
            rs.ry0 = (Tc.y0 + ((int64_t)1 << sh) - 1) >> sh;
            rs.px = px;
            rs.py = py;
            rs.pw = (int)(((rx1 + ((int64_t)1 << px) - 1) >> px) - (rs.rx0 >> px));
            rs.ph = (int)(((ry1 + ((int64_t)1 << py) - 1) >> py) - (rs.ry0 >> py));
            nprec_bands += (int64_t)rs.pw * rs.ph * (int64_t)geo[c][r].bands.size();
            if (nprec_bands > (1 << 22)) { err = "too many precincts"; return TC_E_UNSUPPORTED; }
            for (Band &b : geo[c][r].bands) {
                b.cbw_log2 = xcb;
                b.cbh_log2 = ycb;
                b.ox = (int)((Tc.x0 >> b.level) & ((1 << xcb) - 1));
                b.oy = (int)((Tc.y0 >> b.level) & ((1 << ycb) - 1));
                b.ncbx = b.w > 0 ? ceil_div(b.ox + b.w, 1 << xcb) : 0;
                b.ncby = b.h > 0 ? ceil_div(b.oy + b.h, 1 << ycb) : 0;
            }
            const int ppx = r ? px - 1 : px, ppy = r ? py - 1 : py;
            const int64_t kx0 = rs.rx0 >> px, ky0 = rs.ry0 >> py;
            for (const Band &b : geo[c][r].bands) rs.cb.emplace_back((size_t)b.ncbx * b.ncby);
            rs.prec.resize((size_t)rs.pw * rs.ph);
            for (int q = 0; q < rs.ph; q++)
                for (int p = 0; p < rs.pw; p++) {
                    auto &pbs = rs.prec[(size_t)q * rs.pw + p];
                    for (const Band &b : geo[c][r].bands) {
                        PrecBand pb;
                        // the band and the precinct cell on the band's grid
                        const int64_t bx0 = Tc.x0 >> b.level, by0 = Tc.y0 >> b.level;
                        const int64_t cx0 = std::max(bx0, (kx0 + p) << ppx);
                        const int64_t cx1 = std::min(bx0 + b.w, (kx0 + p + 1) << ppx);
                        const int64_t cy0 = std::max(by0, (ky0 + q) << ppy);
                        const int64_t cy1 = std::min(by0 + b.h, (ky0 + q + 1) << ppy);
                        if (cx0 < cx1 && cy0 < cy1) {
                            const int64_t fx = bx0 >> b.cbw_log2, fy = by0 >> b.cbh_log2;
                            pb.i0 = (int)((cx0 >> b.cbw_log2) - fx);
                            pb.i1 = (int)(((cx1 - 1) >> b.cbw_log2) + 1 - fx);
                            pb.j0 = (int)((cy0 >> b.cbh_log2) - fy);
                            pb.j1 = (int)(((cy1 - 1) >> b.cbh_log2) + 1 - fy);
                            pb.incl = TagTree(pb.i1 - pb.i0, pb.j1 - pb.j0);
                            pb.zbp = TagTree(pb.i1 - pb.i0, pb.j1 - pb.j0);
                        }
                        pb.incl.reset_decoder();
                        pb.zbp.reset_decoder();
                        pbs.push_back(std::move(pb));
                    }
                }
        }
        if ((rc = assign_quant(quant_of(P, &ts, c), P.bits, NL, geo[c], err))) return rc;
        // ROI maxshift (ISO H.1): every band codes shift more bit-planes
        if (const int sh = roi_of(P, &ts, c)) {
            for (int r = 0; r <= NL; r++)
                for (Band &b : geo[c][r].bands) {
                    b.mb += sh;
                    if (b.mb > 31) { err = "ROI shift leaves more than 31 bit-planes"; return TC_E_UNSUPPORTED; }
                }
        }
    }

    // The tile-part bodies are read one after the other as one packet
    // sequence; a packet does not straddle two tile-parts.
    size_t part_i = 0;
    size_t pos = parts.empty() ? len : parts[0].first;
    auto part_end = [&]() { return part_i < parts.size() ? parts[part_i].second : len; };

    std::vector<SegNode> arena;
    std::vector<std::pair<CblkState *, uint32_t>> contrib;  // one packet's blocks and lengths
    // Packed packet headers (PPM / PPT): the headers are read from the
    // tile's packed stream at hpos, the bodies from the tile-parts.
    const bool pk = packed != nullptr;
    size_t hpos = 0;
    // One packet (ISO B.9, B.10): layer, resolution, component, precinct.
    auto read_packet = [&](int layer, int r, int c, int prec) -> int {
        while (part_i < parts.size() && pos >= parts[part_i].second) {
            part_i++;
            if (part_i < parts.size()) pos = parts[part_i].first;
        }
        if (part_i >= parts.size() && !pk) { err = "packet data missing"; return TC_E_CODESTREAM; }
        const size_t pend = part_i < parts.size() ? part_end() : pos;
        if (scod & 2) {  // SOP, in the body
            if (pos + 6 <= pend && cs[pos] == 0xFF && cs[pos + 1] == 0x91) pos += 6;
        }
        const uint8_t *hs = pk ? packed->data() : cs;
        size_t &hp = pk ? hpos : pos;
        const size_t hend = pk ? packed->size() : pend;
        BitReader br(hs, hp, hend);
        const int present = br.get();
        contrib.clear();
        ResState &rs = st[c][r];
        if (present) {
            for (size_t bi = 0; bi < geo[c][r].bands.size(); bi++) {
                const Band &b = geo[c][r].bands[bi];
                PrecBand &pb = rs.prec[prec][bi];
                const int gw = pb.i1 - pb.i0;
                for (int j = pb.j0; j < pb.j1; j++)
                    for (int i = pb.i0; i < pb.i1; i++) {
                        CblkState &cb = rs.cb[bi][(size_t)j * b.ncbx + i];
                        const int leaf = (j - pb.j0) * gw + (i - pb.i0);
                        int inc;
                        if (!cb.included) inc = pb.incl.decode(br, leaf, layer + 1);
                        else inc = br.get();
                        if (br.overrun) { err = "packet header overrun"; return TC_E_CODESTREAM; }
                        if (!inc) continue;
                        if (!cb.included) {
                            const int k = pb.zbp.decode_value(br, leaf, 64);
                            if (k < 0) { err = "bad zero bit-plane tag tree"; return TC_E_CODESTREAM; }
                            cb.zbp = k;
                            cb.included = 1;
                        }
                        const int np = get_num_passes(br);
                        int inc_l = 0;
                        while (br.get()) {
                            if (br.overrun || ++inc_l > 32) { err = "bad Lblock increment"; return TC_E_CODESTREAM; }
                        }
                        cb.lblock += inc_l;
                        const int sty = style[c];
                        if (cb.passes + np > 255) { err = "more than 255 coding passes"; return TC_E_CODESTREAM; }
                        if (!(sty & (TC_CBLK_STYLE_BYPASS | TC_CBLK_STYLE_TERMALL))) {
                            const int nbits = cb.lblock + floorlog2(np);
                            if (nbits > 31) { err = "code-block length field too wide"; return TC_E_CODESTREAM; }
                            const uint32_t Lc = br.get_bits(nbits);
                            if (br.overrun) { err = "packet header overrun"; return TC_E_CODESTREAM; }
                            cb.passes += np;
                            contrib.emplace_back(&cb, Lc);
                            continue;
                        }
                        // Terminated segments: one length per segment the new
                        // passes reach, in Lblock + floorlog2(its new passes)
                        // bits (ISO B.10.7.2); a segment left open continues
                        // in the block's next contribution.
                        uint64_t total = 0;
                        for (int left = np; left > 0;) {
                            const int t = cb.passes;
                            int n = 1;
                            while (n < left && !pass_terminates(sty, t + n - 1)) n++;
                            const int nbits = cb.lblock + floorlog2(n);
                            if (nbits > 31) { err = "code-block length field too wide"; return TC_E_CODESTREAM; }
                            const uint32_t Lc = br.get_bits(nbits);
                            if (br.overrun) { err = "packet header overrun"; return TC_E_CODESTREAM; }
                            if (t == 0 || pass_terminates(sty, t - 1)) cb.seglen.push_back(Lc);
                            else if ((cb.seglen.back() += Lc) < Lc) { err = "codeword segment too long"; return TC_E_CODESTREAM; }
                            total += Lc;
                            cb.passes += n;
                            left -= n;
                        }
                        if (total > 0xFFFFFFFFull) { err = "code-block data too long"; return TC_E_CODESTREAM; }
                        contrib.emplace_back(&cb, (uint32_t)total);
                    }
            }
        }
        br.align();
        if (br.overrun) { err = "packet header overrun"; return TC_E_CODESTREAM; }
        hp = br.pos;
        if (scod & 4) {  // EPH, after the header (in the packed stream when headers are packed)
            if (hp + 2 > hend || hs[hp] != 0xFF || hs[hp + 1] != 0x92) { err = "missing EPH"; return TC_E_CODESTREAM; }
            hp += 2;
        }
        for (auto &cl : contrib) {
            if (pos + cl.second > pend) { err = "code-block data runs past the tile-part"; return TC_E_CODESTREAM; }
            if (cl.second) {
                CblkState &cb = *cl.first;
                const int k = (int)arena.size();
                arena.push_back(SegNode{pos, cl.second, -1});
                if (cb.tail >= 0) arena[cb.tail].next = k;
                else cb.head = k;
                cb.tail = k;
                cb.nseg++;
                cb.bytes += cl.second;
            }
            pos += cl.second;
        }
        return TC_OK;
    };

    // Position-driven orders (ISO B.12.1.3-B.12.1.5) visit a precinct at the
    // first reference-grid position it covers, stepping over the tile by the
    // smallest precinct of any component and resolution.
    auto cdx = [&](int c) -> int64_t { return c < 4 ? P.dx[c] : 1; };
    auto cdy = [&](int c) -> int64_t { return c < 4 ? P.dy[c] : 1; };
    int64_t dx = INT64_MAX, dy = INT64_MAX;
    for (int c = 0; c < C; c++)
        for (int r = 0; r <= NL; r++) {
            dx = std::min<int64_t>(dx, cdx(c) << (st[c][r].px + NL - r));
            dy = std::min<int64_t>(dy, cdy(c) << (st[c][r].py + NL - r));
        }
    // precinct of component c, resolution r that starts at reference-grid
    // position (x, y), or -1 (the component's subsampling scales its grid)
    auto prec_at = [&](int c, int r, int64_t x, int64_t y) -> int {
        const ResState &rs = st[c][r];
        const int sh = NL - r, px = rs.px, py = rs.py;
        const int64_t sx_ = cdx(c) << (px + sh), sy_ = cdy(c) << (py + sh);
        const int64_t pmx = ((int64_t)1 << (px + sh)) - 1, pmy = ((int64_t)1 << (py + sh)) - 1;
        const bool sx = x % sx_ == 0 || (x == T.x0 && ((rs.rx0 << sh) & pmx));
        const bool sy = y % sy_ == 0 || (y == T.y0 && ((rs.ry0 << sh) & pmy));
        if (!sx || !sy) return -1;
        const int64_t ux = cdx(c) << sh, uy = cdy(c) << sh;
        const int64_t kx = (((x + ux - 1) / ux) >> px) - (rs.rx0 >> px);
        const int64_t ky = (((y + uy - 1) / uy) >> py) - (rs.ry0 >> py);
        if (kx < 0 || ky < 0 || kx >= rs.pw || ky >= rs.ph) return -1;
        return (int)(ky * rs.pw + kx);
    };
    auto next = [](int64_t v, int64_t step) { return (v / step + 1) * step; };
    // Progression volumes: the tile's POC, else the main header's, else one
    // volume of everything in COD's order.  A packet (c, r, precinct, layer)
    // is read once, at the first volume that reaches it: done[c][r][k]
    // counts the layers already read (ISO A.6.6, B.12).
    std::vector<PocEntry> vols = !ts.poc.empty() ? ts.poc : P.main.poc;
    if (vols.empty()) vols.push_back(PocEntry{0, 0, L, R, C, prog});
    std::vector<std::vector<std::vector<int>>> done(C, std::vector<std::vector<int>>(R));
    for (int c = 0; c < C; c++)
        for (int r = 0; r < R; r++) done[c][r].assign((size_t)st[c][r].pw * st[c][r].ph, 0);
    auto packet = [&](int l, int r, int c, int k) -> int {
        int &d = done[c][r][k];
        if (l < d) return TC_OK;  // read by an earlier volume
        if (l > d) { err = "progression volumes skip a layer"; return TC_E_CODESTREAM; }
        d++;
        return read_packet(l, r, c, k);
    };
    for (const PocEntry &v : vols) {
        const int lye = std::min(v.lye, L), re = std::min(v.re, R), ce = std::min(v.ce, C);
        const int rs = v.rs, cs0 = v.cs;
        auto layers = [&](int r, int c, int k) -> int {
            for (int l = 0; l < lye; l++)
                if (int e = packet(l, r, c, k)) return e;
            return TC_OK;
        };
        switch (v.prog) {
        case 0:  // LRCP
            for (int l = 0; l < lye; l++) for (int r = rs; r < re; r++) for (int c = cs0; c < ce; c++)
                for (int k = 0; k < st[c][r].pw * st[c][r].ph; k++)
                    if ((rc = packet(l, r, c, k))) return rc;
            break;
        case 1:  // RLCP
            for (int r = rs; r < re; r++) for (int l = 0; l < lye; l++) for (int c = cs0; c < ce; c++)
                for (int k = 0; k < st[c][r].pw * st[c][r].ph; k++)
                    if ((rc = packet(l, r, c, k))) return rc;
            break;
        case 2:  // RPCL
            for (int r = rs; r < re; r++)
                for (int64_t y = T.y0; y < T.y1; y = next(y, dy))
                    for (int64_t x = T.x0; x < T.x1; x = next(x, dx))
                        for (int c = cs0; c < ce; c++) {
                            const int k = prec_at(c, r, x, y);
                            if (k >= 0 && (rc = layers(r, c, k))) return rc;
                        }
            break;
        case 3:  // PCRL
            for (int64_t y = T.y0; y < T.y1; y = next(y, dy))
                for (int64_t x = T.x0; x < T.x1; x = next(x, dx))
                    for (int c = cs0; c < ce; c++)
                        for (int r = rs; r < re; r++) {
                            const int k = prec_at(c, r, x, y);
                            if (k >= 0 && (rc = layers(r, c, k))) return rc;
                        }
            break;
        default:  // CPRL
            for (int c = cs0; c < ce; c++)
                for (int64_t y = T.y0; y < T.y1; y = next(y, dy))
                    for (int64_t x = T.x0; x < T.x1; x = next(x, dx))
                        for (int r = rs; r < re; r++) {
                            const int k = prec_at(c, r, x, y);
                            if (k >= 0 && (rc = layers(r, c, k))) return rc;
                        }
            break;
        }
    }

    // Descriptors, component by component; segments are placed once every
    // tile is read (parse_raw_codestream).
    {
        size_t nb = 0;
        for (int c = 0; c < C; c++)
            for (int r = 0; r < R; r++)
                for (const Band &b : geo[c][r].bands) nb += (size_t)b.ncbx * b.ncby;
        out.desc.reserve(out.desc.size() + nb);
        em.first.reserve(em.first.size() + nb + 1);
        em.segs.reserve(em.segs.size() + arena.size());
    }
    for (int c = 0; c < C; c++)
        for (int r = 0; r < R; r++)
            for (size_t bi = 0; bi < geo[c][r].bands.size(); bi++) {
                const Band &b = geo[c][r].bands[bi];
                std::vector<CblkState> &cbs = st[c][r].cb[bi];
                const int cbw = 1 << b.cbw_log2, cbh = 1 << b.cbh_log2;
                for (int j = 0; j < b.ncby; j++)
                    for (int i = 0; i < b.ncbx; i++) {
                        CblkState &cb = cbs[(size_t)j * b.ncbx + i];
                        tc_cblk_desc d;
                        std::memset(&d, 0, sizeof d);
                        const int cx = std::max(i * cbw - b.ox, 0), cy = std::max(j * cbh - b.oy, 0);
                        d.w = (uint16_t)(std::min((i + 1) * cbw - b.ox, b.w) - cx);
                        d.h = (uint16_t)(std::min((j + 1) * cbh - b.oy, b.h) - cy);
                        d.mb = (uint8_t)b.mb;
                        d.orient = (uint8_t)b.orient;
                        const int cw = (int)(tc[c].x1 - tc[c].x0);
                        d.out_pitch = (uint32_t)cw;
                        d.out_off = coef_off + coff[c] + (uint64_t)(b.y0 + cy) * cw + (uint64_t)(b.x0 + cx);
                        d.step = reversible ? 1.0f : b.step;
                        d.flags = reversible ? 0 : TC_CBLK_IRREVERSIBLE;
                        d.style = (uint8_t)style[c];
                        d.roi_shift = (uint8_t)roi_of(P, &ts, c);
                        em.first.push_back((uint32_t)em.segs.size());
                        if (cb.included && cb.passes > 0) {
                            if (cb.zbp > b.mb) { err = "zero bit-planes exceed Mb"; return TC_E_CODESTREAM; }
                            const int numbps = b.mb - cb.zbp;
                            if (numbps == 0 || cb.passes > 3 * numbps - 2 || cb.passes > 255) {
                                err = "coding pass count exceeds the bit-planes";
                                return TC_E_CODESTREAM;
                            }
                            d.zero_bitplanes = (uint8_t)cb.zbp;
                            d.passes = (uint8_t)cb.passes;
                            if (cb.bytes > 0xFFFFFFFFull) { err = "code-block data too long"; return TC_E_CODESTREAM; }
                            d.seg_len = (uint32_t)cb.bytes;
                            if (cb.nseg > 1) em.multi = true;
                            for (int k = cb.head; k >= 0; k = arena[k].next)
                                em.segs.emplace_back(arena[k].off, arena[k].len);
                            if (style[c] & (TC_CBLK_STYLE_BYPASS | TC_CBLK_STYLE_TERMALL)) {
                                if ((int)cb.seglen.size() != pass_segments(style[c], cb.passes)) {
                                    err = "codeword segments do not match the passes";
                                    return TC_E_CODESTREAM;
                                }
                                em.multi = true;
                                em.tables.push_back({out.desc.size(), (uint32_t)em.tab.size(), (uint32_t)cb.seglen.size()});
                                em.tab.insert(em.tab.end(), cb.seglen.begin(), cb.seglen.end());
                            }
                        } else {
                            d.zero_bitplanes = (uint8_t)b.mb;
                            d.passes = 0;
                        }
                        out.desc.push_back(d);
                    }
            }
    return TC_OK;
}

static int parse_raw_codestream(const uint8_t *cs, size_t len, Parsed &out, std::string &err)
{
    Reader rd{cs, len};
    Params P;
    int rc = parse_main(rd, P, err);
    if (rc) return rc;
    fill_info(P, out.info);
    const size_t ntiles = P.tiles.size();

    // Tile-parts (ISO A.4.2) in codestream order, grouped by tile index Isot:
    // the packet data range of each.  The first tile-part of a tile may carry
    // COD / COC / QCD / QCC for that tile.
    std::vector<std::vector<std::pair<size_t, size_t>>> parts(ntiles);
    std::vector<Scope> tscope(ntiles);
    for (Scope &t : tscope) t.init(P.ncomp);
    // Packed packet headers per tile: PPT segments (Zppt, bytes) from its
    // tile-part headers, or its tile-parts' shares of the PPM stream, which
    // gives each tile-part in codestream order Nppm (32 bits) and then Nppm
    // bytes of headers.
    std::vector<std::vector<std::pair<int, std::vector<uint8_t>>>> ppt(ntiles);
    std::vector<std::vector<uint8_t>> packed(ntiles);
    std::vector<uint8_t> ppm;
    size_t ppm_pos = 0;
    if (!P.ppm.empty()) {
        std::vector<std::pair<int, std::vector<uint8_t>>> segs = P.ppm;
        std::stable_sort(segs.begin(), segs.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
        for (auto &sg : segs) ppm.insert(ppm.end(), sg.second.begin(), sg.second.end());
    }
    for (;;) {
        const uint32_t m = rd.u16();
        if (rd.bad) { err = "truncated codestream"; return TC_E_CODESTREAM; }
        if (m == M_EOC) break;
        if (m != M_SOT) { err = "expected SOT"; return TC_E_CODESTREAM; }
        const size_t sot_pos = rd.pos - 2;
        const uint32_t lsot = rd.u16(), isot = rd.u16(), psot = rd.u32();
        rd.u8();  // TPsot
        rd.u8();  // TNsot
        if (lsot != 10 || isot >= ntiles || (psot && psot < 14)) { err = "bad SOT or tile index"; return TC_E_CODESTREAM; }
        const size_t end = psot ? sot_pos + psot : len;
        if (end > len) { err = "tile-part runs past the codestream"; return TC_E_CODESTREAM; }
        const bool first_part = parts[isot].empty();
        for (;;) {
            const uint32_t mm = rd.u16();
            if (rd.bad || rd.pos > end) { err = "truncated tile-part header"; return TC_E_CODESTREAM; }
            if (mm == M_SOD) break;
            const uint32_t L = rd.u16();
            if (L < 2 || rd.pos - 2 + L > end) { err = "bad tile-part marker"; return TC_E_CODESTREAM; }
            const size_t seg_end = rd.pos - 2 + L;
            if (mm == M_COD || mm == M_COC || mm == M_QCD || mm == M_QCC) {
                if (!first_part) { err = "coding parameters after a tile's first tile-part"; return TC_E_CODESTREAM; }
                if ((rc = read_coding_marker(rd, mm, seg_end, P.ncomp, tscope[isot], err))) return rc;
            } else if (mm == M_POC) {
                if ((rc = read_poc(rd, seg_end, P.ncomp, tscope[isot].poc, err))) return rc;
            } else if (mm == M_PPT) {
                if (!P.ppm.empty()) { err = "PPT with PPM"; return TC_E_CODESTREAM; }
                if (seg_end - rd.pos < 1) { err = "bad PPT"; return TC_E_CODESTREAM; }
                const int z = (int)rd.u8();
                ppt[isot].emplace_back(z, std::vector<uint8_t>(cs + rd.pos, cs + seg_end));
            } else if (mm == M_RGN) {
                if (!first_part) { err = "RGN after a tile's first tile-part"; return TC_E_CODESTREAM; }
                if ((rc = read_rgn(rd, seg_end, P.ncomp, tscope[isot], err))) return rc;
            }
            rd.pos = seg_end;
        }
        if (!ppm.empty()) {
            if (ppm.size() - ppm_pos < 4) { err = "PPM has no headers for a tile-part"; return TC_E_CODESTREAM; }
            const uint32_t n = (uint32_t)ppm[ppm_pos] << 24 | (uint32_t)ppm[ppm_pos + 1] << 16 |
                               (uint32_t)ppm[ppm_pos + 2] << 8 | ppm[ppm_pos + 3];
            ppm_pos += 4;
            if (n > ppm.size() - ppm_pos) { err = "PPM headers run past the PPM data"; return TC_E_CODESTREAM; }
            packed[isot].insert(packed[isot].end(), ppm.begin() + ppm_pos, ppm.begin() + ppm_pos + n);
            ppm_pos += n;
        }
        parts[isot].emplace_back(rd.pos, end);
        rd.pos = end;
        if (rd.pos >= len) break;
    }

    // Tiles one after the other, each with its own coefficient planes.
    out.desc.clear();
    out.own_pool.clear();
    out.tiles.clear();
    Emit em;
    uint64_t coef_off = 0;
    for (size_t t = 0; t < ntiles; t++) {
        const Params::Tile &T = P.tiles[t];
        if (parts[t].empty()) { err = "tile " + std::to_string(t) + " has no tile-part"; return TC_E_CODESTREAM; }
        if (!ppt[t].empty()) {
            std::stable_sort(ppt[t].begin(), ppt[t].end(), [](const auto &a, const auto &b) { return a.first < b.first; });
            for (auto &sg : ppt[t]) packed[t].insert(packed[t].end(), sg.second.begin(), sg.second.end());
        }
        const bool pk = !ppm.empty() || !ppt[t].empty();
        if ((rc = parse_tile(cs, len, P, T, tscope[t], parts[t], coef_off, out, em, err, pk ? &packed[t] : nullptr)))
            return rc;
        tc_tile_info ti;
        ti.x0 = (int32_t)(T.x0 - P.xo);
        ti.y0 = (int32_t)(T.y0 - P.yo);
        ti.w = (int32_t)(T.x1 - T.x0);
        ti.h = (int32_t)(T.y1 - T.y0);
        ti.coef_off = coef_off;
        out.tiles.push_back(ti);
        for (int c = 0; c < P.ncomp; c++) {
            const int64_t dx = c < 4 ? P.dx[c] : 1, dy = c < 4 ? P.dy[c] : 1;
            coef_off += (uint64_t)((T.x1 + dx - 1) / dx - (T.x0 + dx - 1) / dx) *
                        (uint64_t)((T.y1 + dy - 1) / dy - (T.y0 + dy - 1) / dy);
        }
    }
    em.first.push_back((uint32_t)em.segs.size());

    // Segments: in place in the codestream when every block has at most one,
    // else gathered block by block into a pool of the parse's own.
    out.pool_is_cs = !em.multi;
    if (em.multi) {
        uint64_t total = 0;
        for (auto &s : em.segs) total += s.second;
        out.own_pool.reserve(total);
    }
    size_t ti = 0;  // next entry of em.tables
    for (size_t k = 0; k < out.desc.size(); k++) {
        tc_cblk_desc &d = out.desc[k];
        const uint32_t a = em.first[k], b = em.first[k + 1];
        if (ti < em.tables.size() && em.tables[ti].desc == k) {
            // 4-byte aligned table of the segment lengths (uint32 each,
            // little-endian), then the codeword
            const Emit::Table &tb = em.tables[ti++];
            out.own_pool.resize((out.own_pool.size() + 3) & ~size_t(3), 0);
            d.seg_off = out.own_pool.size();
            for (uint32_t i = 0; i < tb.n; i++) {
                const uint32_t v = em.tab[tb.at + i];
                const uint8_t le[4] = {(uint8_t)v, (uint8_t)(v >> 8), (uint8_t)(v >> 16), (uint8_t)(v >> 24)};
                out.own_pool.insert(out.own_pool.end(), le, le + 4);
            }
            for (uint32_t s = a; s < b; s++)
                out.own_pool.insert(out.own_pool.end(), cs + em.segs[s].first, cs + em.segs[s].first + em.segs[s].second);
        } else if (em.multi) {
            d.seg_off = a < b ? out.own_pool.size() : 0;
            for (uint32_t s = a; s < b; s++)
                out.own_pool.insert(out.own_pool.end(), cs + em.segs[s].first, cs + em.segs[s].first + em.segs[s].second);
        } else {
            d.seg_off = a < b ? em.segs[a].first : 0;
        }
    }
    out.info.ncblk = (uint32_t)out.desc.size();
    return TC_OK;
}

// ============================ encoder =======================================

int encode_layout(const tc_encode_params &p, EncodeLayout &L, std::string &err)
{
    const int W = p.width, H = p.height, C = p.ncomp, B = p.bits, NL = p.levels;
    if (W < 1 || H < 1 || W > 65535 || H > 65535 || C < 1 || C > 4 || B < 1 || B > 16 || NL < 0 ||
        NL > 15 || p.cblk_log2 < 2 || p.cblk_log2 > 6 || p.progression < 0 || p.progression > 4) {
        err = "encode parameters out of range";
        return TC_E_ARG;
    }
    if (!p.reversible && !(p.base_step > 0.0)) { err = "base_step must be positive"; return TC_E_ARG; }
    if (p.cblk_style & ~0x3F) { err = "unknown code-block style bits"; return TC_E_ARG; }
    if (p.layers < 0 || p.layers > 64) { err = "layers out of range"; return TC_E_ARG; }
    if (p.packed_headers < 0 || p.packed_headers > 2) { err = "packed_headers out of range"; return TC_E_ARG; }
    if ((p.roi_x1 > p.roi_x0 || p.roi_y1 > p.roi_y0) &&
        (p.roi_x0 < 0 || p.roi_y0 < 0 || p.roi_x1 > W || p.roi_y1 > H || p.roi_x1 <= p.roi_x0 || p.roi_y1 <= p.roi_y0)) {
        err = "ROI outside the image";
        return TC_E_ARG;
    }
    // Per component: code-block size (COC when it differs from COD), step
    // multiplier (QCC when it differs from QCD) and subsampling (SIZ).
    for (int c = 0; c < C; c++) {
        L.cblk[c] = p.comp_cblk_log2[c] > 0 ? p.comp_cblk_log2[c] : p.cblk_log2;
        L.scale[c] = p.comp_step_scale[c] > 0.0 ? p.comp_step_scale[c] : 1.0;
        if (L.cblk[c] < 2 || L.cblk[c] > 6) { err = "code-block size out of range"; return TC_E_ARG; }
        L.dx[c] = p.comp_dx[c] > 0 ? p.comp_dx[c] : 1;
        L.dy[c] = p.comp_dy[c] > 0 ? p.comp_dy[c] : 1;
        if (L.dx[c] > 255 || L.dy[c] > 255) { err = "subsampling out of range"; return TC_E_ARG; }
        L.cw[c] = (W + L.dx[c] - 1) / L.dx[c];
        L.ch[c] = (H + L.dy[c] - 1) / L.dy[c];
        L.coff[c + 1] = L.coff[c] + (size_t)L.cw[c] * L.ch[c];
    }
    if (p.mct && C >= 3 && (L.cw[1] != L.cw[0] || L.cw[2] != L.cw[0] || L.ch[1] != L.ch[0] || L.ch[2] != L.ch[0])) {
        err = "the colour transform needs components 0-2 at one size";
        return TC_E_ARG;
    }
    L.geo.assign(C, {});
    for (int c = 0; c < C; c++) L.geo[c] = make_geometry(L.cw[c], L.ch[c], NL, L.cblk[c], L.cblk[c]);
    // Quantisation exponent / mantissa / step per band (ISO E.1).
    for (int c = 0; c < C; c++)
        for (int r = 0; r <= NL; r++)
            for (Band &b : L.geo[c][r].bands) {
                const int rb = B + band_gain_log2(b.orient);
                if (p.reversible) {
                    b.eps = rb;
                    b.mu = 0;
                    b.step = 1.0f;
                } else {
                    const double delta =
                        L.scale[c] * p.base_step * std::ldexp(1.0, B) / subband_norm(true, b.level, b.orient);
                    int e = rb - (int)std::floor(std::log2(delta));
                    int m = (int)std::lround((delta / std::ldexp(1.0, rb - e) - 1.0) * 2048.0);
                    if (m >= 2048) { m = 0; e--; }
                    if (m < 0) m = 0;
                    if (e < 0 || e > 31) { err = "quantisation step out of range"; return TC_E_ARG; }
                    b.eps = e;
                    b.mu = m;
                    b.step = (float)std::ldexp(1.0 + m / 2048.0, rb - e);
                }
            }
    // Code-blocks in packet order.
    L.jobs.clear();
    for (int c = 0; c < C; c++)
        for (int r = 0; r <= NL; r++)
            for (int bi = 0; bi < (int)L.geo[c][r].bands.size(); bi++) {
                const Band &b = L.geo[c][r].bands[bi];
                for (int j = 0; j < b.ncby; j++)
                    for (int i = 0; i < b.ncbx; i++) L.jobs.push_back({c, r, bi, i, j});
            }
    return TC_OK;
}

// The host encoder: colour transform and DWT on the CPU (double precision
// for 9/7), deadzone quantisation, Tier-1 per code-block, then
// encode_assemble.
int encode_codestream(const tc_encode_params &p, const void *planes, std::vector<uint8_t> &out,
                      std::string &err)
{
    EncodeLayout L;
    int rc = encode_layout(p, L, err);
    if (rc) return rc;
    const int C = p.ncomp, B = p.bits, NL = p.levels;
    const bool mct = p.mct && C >= 3;
    const int threads = p.threads;
    const size_t np = (size_t)L.cw[0] * L.ch[0];  // components 0-2 under a colour transform
    const size_t ntot = L.coff[C];
    const bool wide = B > 8;

    std::vector<int32_t> ip;
    std::vector<double> dp;
    const bool sgn = p.is_signed != 0;
    auto sample = [&](size_t i) -> int32_t {
        if (sgn) return wide ? ((const int16_t *)planes)[i] : ((const int8_t *)planes)[i];
        return wide ? ((const uint16_t *)planes)[i] : ((const uint8_t *)planes)[i];
    };
    const int32_t dc = sgn ? 0 : 1 << (B - 1);  // ISO G.1.2: unsigned samples only
    if (p.reversible) {
        ip.resize(ntot);
        for (size_t i = 0; i < ntot; i++) ip[i] = sample(i) - dc;
        if (mct)
            for (size_t i = 0; i < np; i++) {
                const int32_t r = ip[i], g = ip[np + i], b = ip[2 * np + i];
                ip[i] = (r + 2 * g + b) >> 2;
                ip[np + i] = b - g;
                ip[2 * np + i] = r - g;
            }
        for (int c = 0; c < C; c++)
            fwd_plane_pitch(ip.data() + L.coff[c], L.cw[c], L.ch[c], (size_t)L.cw[c], NL, fwd53_line, threads);
    } else {
        dp.resize(ntot);
        for (size_t i = 0; i < ntot; i++) dp[i] = (double)(sample(i) - dc);
        if (mct)
            for (size_t i = 0; i < np; i++) {
                const double R = dp[i], G = dp[np + i], Bl = dp[2 * np + i];
                dp[i] = 0.299 * R + 0.587 * G + 0.114 * Bl;
                dp[np + i] = -0.16875 * R - 0.33126 * G + 0.5 * Bl;
                dp[2 * np + i] = 0.5 * R - 0.41869 * G - 0.08131 * Bl;
            }
        for (int c = 0; c < C; c++)
            fwd_plane_pitch(dp.data() + L.coff[c], L.cw[c], L.ch[c], (size_t)L.cw[c], NL, fwd97_line, threads);
    }

    // Quantised coefficients.
    std::vector<int32_t> q(ntot);
    for (int c = 0; c < C; c++)
        for (int r = 0; r <= NL; r++)
            for (const Band &b : L.geo[c][r].bands)
                for (int y = b.y0; y < b.y0 + b.h; y++)
                    for (int x = b.x0; x < b.x0 + b.w; x++) {
                        const size_t i = L.coff[c] + (size_t)y * L.cw[c] + x;
                        int32_t v;
                        if (p.reversible) {
                            v = ip[i];
                        } else {
                            const double a = std::fabs(dp[i]) / (double)b.step;
                            v = (int32_t)std::floor(a);
                            if (dp[i] < 0) v = -v;
                        }
                        q[i] = v;
                    }

    // ROI maxshift (ISO Annex H): coefficients whose band cell (scaled by
    // the band's level) meets the region are shifted up by s, so that every
    // region bit lies above every background bit; the decoder needs no mask.
    // s is one more than the bit count of the largest background magnitude:
    // ISO asks 2^s above the background, and OpenJPEG's decoder compares its
    // half-bit-scaled values with 2^s, so it needs 2^(s-1) above it.
    std::vector<uint8_t> in_roi;
    const bool roi = p.roi_x1 > p.roi_x0 && p.roi_y1 > p.roi_y0;
    if (roi) {
        in_roi.assign(ntot, 0);
        for (int c = 0; c < C; c++) {
            const int64_t rx0 = p.roi_x0 / L.dx[c], ry0 = p.roi_y0 / L.dy[c];
            const int64_t rx1 = (p.roi_x1 + L.dx[c] - 1) / L.dx[c], ry1 = (p.roi_y1 + L.dy[c] - 1) / L.dy[c];
            int bg = 0;
            for (int r = 0; r <= NL; r++)
                for (const Band &b : L.geo[c][r].bands)
                    for (int y = 0; y < b.h; y++)
                        for (int x = 0; x < b.w; x++) {
                            const size_t i = L.coff[c] + (size_t)(b.y0 + y) * L.cw[c] + b.x0 + x;
                            const bool in = ((int64_t)(x + 1) << b.level) > rx0 && ((int64_t)x << b.level) < rx1 &&
                                            ((int64_t)(y + 1) << b.level) > ry0 && ((int64_t)y << b.level) < ry1;
                            in_roi[i] = in;
                            if (!in) bg = std::max(bg, 32 - __builtin_clz((uint32_t)std::abs(q[i]) | 1u) - (q[i] == 0));
                        }
            L.roi[c] = bg ? bg + 1 : 0;
            const int sh = L.roi[c];
            if (sh)
                for (size_t i = L.coff[c]; i < L.coff[c + 1]; i++)
                    if (in_roi[i]) q[i] = q[i] < 0 ? -(-q[i] << sh) : q[i] << sh;
        }
    }

    // Tier-1: every code-block with all passes; the codeword does not
    // depend on Mb, so the blocks are coded before the guard bits are known.
    std::vector<CodedBlock> coded(L.jobs.size());
    std::vector<std::vector<uint8_t>> words(L.jobs.size());
    std::vector<std::vector<std::pair<uint32_t, int>>> segs(L.jobs.size());
    const int style = p.cblk_style;
    const bool segmented = style & (TC_CBLK_STYLE_BYPASS | TC_CBLK_STYLE_TERMALL);
    std::atomic<int> fail{0};
    parallel_for((int)L.jobs.size(), threads, [&](int k) {
        const EncodeLayout::Job &jb = L.jobs[k];
        const Band &b = L.geo[jb.c][jb.r].bands[jb.bi];
        const int cx = jb.i << b.cbw_log2, cy = jb.j << b.cbh_log2;
        const int bw = std::min(1 << b.cbw_log2, b.w - cx), bh = std::min(1 << b.cbh_log2, b.h - cy);
        int32_t blk[64 * 64];
        uint32_t plain = 0;  // largest magnitude before the ROI shift
        for (int y = 0; y < bh; y++)
            for (int x = 0; x < bw; x++) {
                const size_t i = L.coff[jb.c] + (size_t)(b.y0 + cy + y) * L.cw[jb.c] + b.x0 + cx + x;
                blk[y * bw + x] = q[i];
                const uint32_t a = (uint32_t)std::abs(q[i]);
                plain = std::max(plain, roi && in_roi[i] ? a >> L.roi[jb.c] : a);
            }
        coded[k].numbps_plain = plain ? 32 - __builtin_clz(plain) : 0;
        int zbp = 0;
        if (t1_encode_block(blk, bw, bh, b.orient, 31, 0, words[k], &coded[k].passes, &zbp, style,
                            segmented ? &segs[k] : nullptr))
            fail = 1;
        coded[k].numbps = 31 - zbp;
        coded[k].data = words[k].data();
        coded[k].len = (uint32_t)words[k].size();
        coded[k].seg = segs[k].data();
        coded[k].nseg = (int)segs[k].size();
    });
    if (fail) { err = "Tier-1 encoding failed"; return TC_E_ARG; }
    return encode_assemble(p, L, coded, out, err);
}

int encode_assemble(const tc_encode_params &p, EncodeLayout &L, const std::vector<CodedBlock> &coded,
                    std::vector<uint8_t> &out, std::string &err)
{
    const int W = p.width, H = p.height, C = p.ncomp, B = p.bits, NL = p.levels;
    const bool mct = p.mct && C >= 3;
    const bool sgn = p.is_signed != 0;
    auto &geo = L.geo;
    const int *cblk = L.cblk;
    const double *scale = L.scale;
    const auto &jobs = L.jobs;
    if (coded.size() != jobs.size()) { err = "coded block count does not match the layout"; return TC_E_ARG; }
    // Guard bits (ISO E.1): enough for every band's largest magnitude.
    std::vector<std::vector<std::vector<int>>> band_bps(C, std::vector<std::vector<int>>(NL + 1));
    for (int c = 0; c < C; c++)
        for (int r = 0; r <= NL; r++) band_bps[c][r].assign(geo[c][r].bands.size(), 0);
    for (size_t k = 0; k < jobs.size(); k++) {
        int &m = band_bps[jobs[k].c][jobs[k].r][jobs[k].bi];
        m = std::max(m, coded[k].numbps_plain >= 0 ? coded[k].numbps_plain : coded[k].numbps);
    }
    int need_guard = 1;
    for (int c = 0; c < C; c++)
        for (int r = 0; r <= NL; r++)
            for (size_t bi = 0; bi < geo[c][r].bands.size(); bi++)
                need_guard = std::max(need_guard, band_bps[c][r][bi] - geo[c][r].bands[bi].eps + 1);
    int G = p.guard_bits > 0 ? p.guard_bits : std::max(2, need_guard);
    if (G < need_guard || G > 7) { err = "guard bits cannot hold the coefficient range"; return TC_E_ARG; }
    for (int c = 0; c < C; c++)
        for (int r = 0; r <= NL; r++)
            for (Band &b : geo[c][r].bands) {
                b.mb = G + b.eps - 1;
                if (b.mb + L.roi[c] > 31) { err = "more than 31 magnitude bit-planes"; return TC_E_ARG; }
            }
    std::vector<int> zbps(jobs.size());
    for (size_t k = 0; k < jobs.size(); k++) {
        zbps[k] = geo[jobs[k].c][jobs[k].r].bands[jobs[k].bi].mb + L.roi[jobs[k].c] - coded[k].numbps;
        if (zbps[k] < 0) { err = "a block codes more bit-planes than its band"; return TC_E_ARG; }
    }

    // Index jobs by (c, r, bi) for the packet writer.
    std::vector<std::vector<std::vector<int>>> first(C, std::vector<std::vector<int>>(NL + 1));
    for (size_t k = 0; k < jobs.size(); k++) {
        auto &v = first[jobs[k].c][jobs[k].r];
        if ((int)v.size() <= jobs[k].bi) v.resize(jobs[k].bi + 1, -1);
        if (v[jobs[k].bi] < 0) v[jobs[k].bi] = (int)k;
    }

    // Main header, then the single tile-part: its length is patched in once
    // the packets are written straight into `out`.
    size_t total = 0;
    for (const CodedBlock &cb : coded) total += cb.len;
    out.clear();
    out.reserve(1024 + total + 8 * jobs.size());
    Writer wr{out};
    wr.u16(M_SOC);
    wr.u16(M_SIZ);
    wr.u16(38 + 3 * C);
    wr.u16(0);
    wr.u32(W); wr.u32(H); wr.u32(0); wr.u32(0);
    wr.u32(W); wr.u32(H); wr.u32(0); wr.u32(0);
    wr.u16(C);
    for (int c = 0; c < C; c++) { wr.u8((B - 1) | (sgn ? 0x80 : 0)); wr.u8(L.dx[c]); wr.u8(L.dy[c]); }
    wr.u16(M_COD);
    wr.u16(12);
    wr.u8(0);                              // Scod: default precincts, no SOP/EPH
    wr.u8(p.progression);                  // progression order
    wr.u16(std::max(1, p.layers));         // layers
    wr.u8(mct ? 1 : 0);
    wr.u8(NL);
    wr.u8(p.cblk_log2 - 2);
    wr.u8(p.cblk_log2 - 2);
    wr.u8(p.cblk_style);                   // code-block style
    wr.u8(p.reversible ? 1 : 0);
    // COC for components whose code-block size differs from COD's
    for (int c = 0; c < C; c++) {
        if (cblk[c] == p.cblk_log2) continue;
        wr.u16(M_COC);
        wr.u16(9);
        wr.u8(c);                          // Ccoc
        wr.u8(0);                          // Scoc: default precincts
        wr.u8(NL);
        wr.u8(cblk[c] - 2);
        wr.u8(cblk[c] - 2);
        wr.u8(p.cblk_style);
        wr.u8(p.reversible ? 1 : 0);
    }
    const int nbands = 3 * NL + 1;
    // QCD with component 0's steps, QCC for components whose steps differ
    auto write_steps = [&](int c) {
        if (p.reversible) wr.u8((G << 5) | 0);
        else wr.u8((G << 5) | 2);
        for (int r = 0; r <= NL; r++)
            for (const Band &b : geo[c][r].bands) {
                if (p.reversible) wr.u8(b.eps << 3);
                else wr.u16((b.eps << 11) | b.mu);
            }
    };
    const int qbytes = p.reversible ? nbands : 2 * nbands;
    wr.u16(M_QCD);
    wr.u16(3 + qbytes);
    write_steps(0);
    for (int c = 1; c < C; c++) {
        if (scale[c] == scale[0]) continue;
        wr.u16(M_QCC);
        wr.u16(4 + qbytes);
        wr.u8(c);                          // Cqcc
        write_steps(c);
    }
    // Packets go to `body`; their headers too, or to `hdrs` when they are
    // packed into PPT / PPM marker segments (p.packed_headers 1 / 2).
    std::vector<uint8_t> body, hdrs;
    body.reserve(total + 8 * jobs.size());
    std::vector<uint8_t> &hdst = p.packed_headers ? hdrs : body;
    // Quality layers: block k's passes [lp(k, l), lp(k, l + 1)) go into
    // layer l.  A codeword segment that a layer boundary cuts is split by
    // bytes in proportion to its passes, so a decoder given every layer
    // reads the whole codeword (the harness computes no rate-distortion
    // truncation points).
    const int NLY = std::max(1, p.layers);
    auto lp = [&](size_t k, int l) { return (int)((int64_t)coded[k].passes * l / NLY); };
    // bytes of block k's codeword that its first t passes span
    auto bytes_at = [&](size_t k, int t) -> uint32_t {
        const CodedBlock &cd = coded[k];
        if (t >= cd.passes) return cd.len;
        const std::pair<uint32_t, int> whole(cd.len, cd.passes);
        const std::pair<uint32_t, int> *sg = cd.nseg ? cd.seg : &whole;
        const int ns = cd.nseg ? cd.nseg : 1;
        uint32_t b = 0;
        int a = 0;  // first pass of segment s
        for (int s = 0; s < ns; s++) {
            if (t < a + sg[s].second)
                return b + (uint32_t)((uint64_t)sg[s].first * (uint64_t)(t - a) / (uint64_t)sg[s].second);
            b += sg[s].first;
            a += sg[s].second;
        }
        return b;
    };
    // Per band: inclusion (first layer with passes) and zero bit-plane tag
    // trees; per block: Lblock and whether it was included.
    std::vector<std::vector<std::vector<TagTree>>> incl(C), ztree(C);
    std::vector<int> lblock(jobs.size(), 3);
    std::vector<uint8_t> included(jobs.size(), 0);
    for (int c = 0; c < C; c++) {
        incl[c].resize(NL + 1);
        ztree[c].resize(NL + 1);
        for (int r = 0; r <= NL; r++)
            for (int bi = 0; bi < (int)geo[c][r].bands.size(); bi++) {
                const Band &b = geo[c][r].bands[bi];
                const int n = b.ncbx * b.ncby;
                incl[c][r].emplace_back(std::max(b.ncbx, 1), std::max(b.ncby, 1));
                ztree[c][r].emplace_back(std::max(b.ncbx, 1), std::max(b.ncby, 1));
                if (n == 0) continue;
                const int k0 = first[c][r][bi];
                std::vector<int> iv(n), zv(n);
                for (int i = 0; i < n; i++) {
                    int fl = NLY;  // never included
                    for (int l = 0; l < NLY; l++)
                        if (lp(k0 + i, l + 1) > lp(k0 + i, l)) { fl = l; break; }
                    iv[i] = fl;
                    zv[i] = zbps[k0 + i];
                }
                incl[c][r][bi].set_leaves(iv);
                ztree[c][r][bi].set_leaves(zv);
            }
    }
    std::vector<uint8_t> hdr;
    auto write_packet = [&](int l, int r, int c) {
        hdr.clear();
        BitWriter bw(hdr);
        bool any = false;
        for (int bi = 0; bi < (int)geo[c][r].bands.size(); bi++) {
            const Band &b = geo[c][r].bands[bi];
            if (b.ncbx * b.ncby == 0) continue;
            const int k0 = first[c][r][bi];
            for (int i = 0; i < b.ncbx * b.ncby; i++) any |= lp(k0 + i, l + 1) > lp(k0 + i, l);
        }
        if (!any) {
            bw.put(0);
            bw.flush();
            hdst.insert(hdst.end(), hdr.begin(), hdr.end());
            return;
        }
        bw.put(1);
        std::vector<std::pair<uint32_t, uint32_t>> ranges;  // byte ranges of the blocks' codewords
        std::vector<std::pair<uint32_t, int>> chunks;
        for (int bi = 0; bi < (int)geo[c][r].bands.size(); bi++) {
            const Band &b = geo[c][r].bands[bi];
            const int n = b.ncbx * b.ncby;
            if (n == 0) continue;
            const int k0 = first[c][r][bi];
            for (int i = 0; i < n; i++) {
                const size_t k = (size_t)k0 + i;
                const CodedBlock &cd = coded[k];
                const int t0 = lp(k, l), t1 = lp(k, l + 1);
                if (!included[k]) incl[c][r][bi].encode(bw, i, l + 1);
                else bw.put(t1 > t0);
                if (t1 == t0) continue;
                if (!included[k]) {
                    ztree[c][r][bi].encode(bw, i, zbps[k] + 1);
                    included[k] = 1;
                }
                put_num_passes(bw, t1 - t0);
                // The new passes in codeword-segment chunks (cut at the
                // segments' last passes), one Lblock increment, then each
                // chunk's length in Lblock + floorlog2(its passes) bits
                // (ISO B.10.7).
                chunks.clear();
                if (!cd.nseg) {
                    chunks.emplace_back(bytes_at(k, t1) - bytes_at(k, t0), t1 - t0);
                } else {
                    int a = 0;
                    for (int s = 0; s < cd.nseg; s++) {
                        const int e = a + cd.seg[s].second;
                        const int u0 = std::max(a, t0), u1 = std::min(e, t1);
                        if (u0 < u1) chunks.emplace_back(bytes_at(k, u1) - bytes_at(k, u0), u1 - u0);
                        a = e;
                    }
                }
                int incr = 0;
                for (auto &ch : chunks)
                    while (ch.first >= (1u << (lblock[k] + incr + floorlog2(ch.second)))) incr++;
                for (int t = 0; t < incr; t++) bw.put(1);
                bw.put(0);
                lblock[k] += incr;
                for (auto &ch : chunks) bw.put_bits(ch.first, lblock[k] + floorlog2(ch.second));
                ranges.emplace_back(bytes_at(k, t0), bytes_at(k, t1));
                (void)cd;
            }
        }
        bw.flush();
        hdst.insert(hdst.end(), hdr.begin(), hdr.end());
        size_t bi = 0;
        for (int bb = 0; bb < (int)geo[c][r].bands.size(); bb++) {
            const Band &b = geo[c][r].bands[bb];
            const int n = b.ncbx * b.ncby;
            if (n == 0) continue;
            const int k0 = first[c][r][bb];
            for (int i = 0; i < n; i++) {
                const size_t k = (size_t)k0 + i;
                if (lp(k, l + 1) == lp(k, l)) continue;
                const auto &rg = ranges[bi++];
                body.insert(body.end(), coded[k].data + rg.first, coded[k].data + rg.second);
            }
        }
    };
    // One precinct per resolution, all at the origin: LRCP visits (l, r, c),
    // RLCP (r, l, c), RPCL (r, c, l), PCRL and CPRL (c, r, l).
    switch (p.progression) {
    case 0:
        for (int l = 0; l < NLY; l++)
            for (int r = 0; r <= NL; r++)
                for (int c = 0; c < C; c++) write_packet(l, r, c);
        break;
    case 1:
        for (int r = 0; r <= NL; r++)
            for (int l = 0; l < NLY; l++)
                for (int c = 0; c < C; c++) write_packet(l, r, c);
        break;
    case 2:
        for (int r = 0; r <= NL; r++)
            for (int c = 0; c < C; c++)
                for (int l = 0; l < NLY; l++) write_packet(l, r, c);
        break;
    default:
        for (int c = 0; c < C; c++)
            for (int r = 0; r <= NL; r++)
                for (int l = 0; l < NLY; l++) write_packet(l, r, c);
        break;
    }

    // Packed packet headers (ISO A.7.4-A.7.5): PPM in the main header holds,
    // for the one tile-part, Nppm and the headers; PPT in the tile-part
    // header holds the headers.  Each marker segment carries at most 65532
    // bytes after its index.
    auto put_packed = [&](uint32_t marker, const std::vector<uint8_t> &data) {
        size_t at = 0;
        int z = 0;
        do {
            const size_t n = std::min<size_t>(data.size() - at, 65532);
            wr.u16(marker);
            wr.u16((uint32_t)(n + 3));
            wr.u8(z++ & 0xFF);
            out.insert(out.end(), data.begin() + at, data.begin() + at + n);
            at += n;
        } while (at < data.size());
    };
    if (p.packed_headers == 2) {
        std::vector<uint8_t> ippm = {(uint8_t)(hdrs.size() >> 24), (uint8_t)(hdrs.size() >> 16),
                                     (uint8_t)(hdrs.size() >> 8), (uint8_t)hdrs.size()};
        ippm.insert(ippm.end(), hdrs.begin(), hdrs.end());
        put_packed(M_PPM, ippm);
    }
    // RGN: the maxshift value of each component with a region (ISO A.6.3)
    for (int c = 0; c < C; c++) {
        if (!L.roi[c]) continue;
        wr.u16(M_RGN);
        wr.u16(5);
        wr.u8(c);                          // Crgn
        wr.u8(0);                          // Srgn: maxshift
        wr.u8(L.roi[c]);                   // SPrgn
    }
    const size_t sot = out.size();
    wr.u16(M_SOT);
    wr.u16(10);
    wr.u16(0);
    wr.u32(0);  // Psot, below
    wr.u8(0);
    wr.u8(1);
    if (p.packed_headers == 1) put_packed(M_PPT, hdrs);
    wr.u16(M_SOD);
    out.insert(out.end(), body.begin(), body.end());
    const uint32_t psot = (uint32_t)(out.size() - sot);
    out[sot + 6] = (uint8_t)(psot >> 24);
    out[sot + 7] = (uint8_t)(psot >> 16);
    out[sot + 8] = (uint8_t)(psot >> 8);
    out[sot + 9] = (uint8_t)psot;
    wr.u16(M_EOC);
    return TC_OK;
}

}  // namespace tc

namespace tc {

// ---- JP2 file format (ISO 15444-1 Annex I; the reference's
//      jp2_parse_boxes, boxes.c:265-307, reached from Decoder::decode for
//      .jp2 files, Decoder.cpp:121-125) ------------------------------------
//
// A JP2 file is a sequence of boxes: a 4-byte big-endian length LBox (1: an
// 8-byte length XLBox follows; 0: the box runs to the end of the file), a
// 4-byte type, then the content.  The decoder needs the signature box, the
// file type box (brand or compatibility list "jp2 "), the header superbox
// with its image header box, and the first contiguous codestream box, whose
// content is the codestream.

namespace {

constexpr uint32_t kBoxSig = 0x6A502020u, kBoxFtyp = 0x66747970u, kBoxJp2h = 0x6A703268u,
                   kBoxIhdr = 0x69686472u, kBoxJp2c = 0x6A703263u, kSigContent = 0x0D0A870Au,
                   kBrandJp2 = 0x6A703220u;

uint32_t be32(const uint8_t *p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

struct Box {
    uint32_t type = 0;
    size_t body = 0, end = 0;  // content [body, end) of the buffer
};

// The box starting at `pos` of d[0..len); false when it does not fit.
bool next_box(const uint8_t *d, size_t len, size_t pos, Box &b)
{
    if (len < 8 || pos > len - 8) return false;
    uint64_t lbox = be32(d + pos);
    b.type = be32(d + pos + 4);
    size_t hdr = 8;
    if (lbox == 1) {
        if (pos > len - 16) return false;
        lbox = (uint64_t)be32(d + pos + 8) << 32 | be32(d + pos + 12);
        hdr = 16;
    } else if (lbox == 0) {
        lbox = len - pos;
    }
    if (lbox < hdr || lbox > len - pos) return false;
    b.body = pos + hdr;
    b.end = pos + (size_t)lbox;
    return true;
}

struct Jp2Header {
    bool have = false;
    uint32_t width = 0, height = 0, ncomp = 0;
};

// Locates the codestream of a JP2 file; a buffer that starts with the SOC
// marker is a codestream already (offset 0).
int locate_codestream(const uint8_t *d, size_t len, size_t &off, size_t &n, Jp2Header &ih, std::string &err)
{
    off = 0;
    n = len;
    if (len >= 2 && d[0] == 0xFF && d[1] == 0x4F) return TC_OK;
    Box b;
    if (!next_box(d, len, 0, b) || b.type != kBoxSig || b.end - b.body != 4 || be32(d + b.body) != kSigContent) {
        err = "neither a JPEG 2000 codestream (SOC) nor a JP2 file (signature box)";
        return TC_E_CODESTREAM;
    }
    bool ftyp_ok = false;
    for (size_t pos = b.end; pos < len;) {
        if (!next_box(d, len, pos, b)) {
            err = "truncated JP2 box";
            return TC_E_CODESTREAM;
        }
        if (b.type == kBoxFtyp) {
            for (size_t q = b.body; q + 4 <= b.end; q += 4)
                if ((q == b.body || q >= b.body + 8) && be32(d + q) == kBrandJp2) ftyp_ok = true;
        } else if (b.type == kBoxJp2h) {
            Box c;
            for (size_t q = b.body; q < b.end; q = c.end) {
                if (!next_box(d, b.end, q, c)) {
                    err = "truncated box in the JP2 header";
                    return TC_E_CODESTREAM;
                }
                if (c.type == kBoxIhdr && c.end - c.body >= 14) {
                    ih.have = true;
                    ih.height = be32(d + c.body);
                    ih.width = be32(d + c.body + 4);
                    ih.ncomp = (uint32_t)d[c.body + 8] << 8 | d[c.body + 9];
                }
            }
        } else if (b.type == kBoxJp2c) {
            if (!ftyp_ok) {
                err = "JP2 file without a jp2 file type box before its codestream";
                return TC_E_CODESTREAM;
            }
            off = b.body;
            n = b.end - b.body;
            return TC_OK;
        }
        pos = b.end;
    }
    err = "JP2 file without a codestream box";
    return TC_E_CODESTREAM;
}

int check_header(const Jp2Header &ih, const tc_image_info &info, std::string &err)
{
    if (ih.have && (ih.width != (uint32_t)info.width || ih.height != (uint32_t)info.height ||
                    ih.ncomp != (uint32_t)info.ncomp)) {
        err = "the JP2 image header disagrees with the codestream's SIZ marker";
        return TC_E_CODESTREAM;
    }
    return TC_OK;
}

}  // namespace

int read_header(const uint8_t *cs, size_t len, tc_image_info &info, std::string &err)
{
    size_t off, n;
    Jp2Header ih;
    int rc = locate_codestream(cs, len, off, n, ih, err);
    if (rc) return rc;
    if ((rc = read_raw_header(cs + off, n, info, err))) return rc;
    return check_header(ih, info, err);
}

int parse_codestream(const uint8_t *cs, size_t len, Parsed &out, std::string &err)
{
    size_t off, n;
    Jp2Header ih;
    int rc = locate_codestream(cs, len, off, n, ih, err);
    if (rc) return rc;
    if ((rc = parse_raw_codestream(cs + off, n, out, err))) return rc;
    if ((rc = check_header(ih, out.info, err))) return rc;
    // Segments of a single-layer stream are read in place: make their offsets
    // count from the start of the file.
    if (off && out.pool_is_cs)
        for (tc_cblk_desc &d : out.desc) d.seg_off += off;
    return TC_OK;
}

}  // namespace tc
