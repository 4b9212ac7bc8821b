// j2k_host.h -- host-side codestream geometry, parser and harness encoder
// shared by the C ABI implementation.  Host code only (no CUDA types).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "tc_j2k.h"

namespace tc {

// One subband of a tile-component, positioned in the component's Mallat
// plane.  Geometry follows ISO B.5 for a tile anchored at the origin; the
// reference builds the same tree in init_resolution_lvls / init_subbands /
// init_codeblocks (codestream_image.c:96-230).
struct Band {
    int orient = 0;       // 0 LL, 1 HL, 2 LH, 3 HH
    int level = 0;        // decomposition level n_b (LL_N: N)
    int x0 = 0, y0 = 0;   // position in the Mallat plane
    int w = 0, h = 0;
    int cbw_log2 = 6, cbh_log2 = 6;
    int ncbx = 0, ncby = 0;
    // offset of the band's first sample inside its first code-block: the
    // code-block grid is anchored at the reference grid's origin (ISO B.7),
    // so a tile that does not start on a block boundary has a narrower
    // first block.  Block i spans [max(i*cbw - ox, 0), min((i+1)*cbw - ox, w)).
    int ox = 0, oy = 0;
    int eps = 0, mu = 0;  // quantisation exponent / mantissa
    int mb = 0;           // magnitude bit-planes
    float step = 1.0f;    // irreversible step
};

struct Resolution {
    int w = 0, h = 0;
    std::vector<Band> bands;  // r = 0: LL; r > 0: HL, LH, HH
};

// Level sizes ws[d], hs[d] of the LL band after d decompositions.
void level_sizes(int w, int h, int levels, std::vector<int> &ws, std::vector<int> &hs);
std::vector<Resolution> make_geometry(int w, int h, int levels, int xcb, int ycb);

// log2 of the subband gain (ISO E.1: LL 0, HL/LH 1, HH 2).
inline int band_gain_log2(int orient) { return orient == 0 ? 0 : (orient == 3 ? 2 : 1); }

// Synthesis basis L2 norm of a subband (9/7 when wavelet97, else 5/3).
double subband_norm(bool wavelet97, int level, int orient);

// ---- MQ encoder / Tier-1 encoder (harness) ---------------------------------
// `style`: code-block style bits (TC_CBLK_STYLE_*); `segments`, when given,
// receives each terminated codeword segment's length and pass count.
int t1_encode_block(const int32_t *coef, int w, int h, int orient, int mb, int passes,
                    std::vector<uint8_t> &out, int *passes_out, int *zero_bitplanes, int style = 0,
                    std::vector<std::pair<uint32_t, int>> *segments = nullptr);

// ---- parser -----------------------------------------------------------------
struct Parsed {
    tc_image_info info{};
    std::vector<tc_cblk_desc> desc;
    std::vector<uint8_t> own_pool;  // used when blocks have several segments
    bool pool_is_cs = true;
    std::vector<tc_tile_info> tiles;  // info.ntiles entries
};
// cs: a raw codestream (starts with SOC) or a JP2 file, whose first
// codestream box is decoded; segment offsets count from the start of `cs`.
int parse_codestream(const uint8_t *cs, size_t len, Parsed &out, std::string &err);
int read_header(const uint8_t *cs, size_t len, tc_image_info &info, std::string &err);

// ---- encoder ------------------------------------------------------------------
// Layout of a codestream to encode: per component the code-block size, step
// multiplier and subband geometry with its quantisation (eps, mu, step),
// and the code-blocks in packet order.
struct EncodeLayout {
    int cblk[4] = {6, 6, 6, 6};
    double scale[4] = {1, 1, 1, 1};
    int dx[4] = {1, 1, 1, 1}, dy[4] = {1, 1, 1, 1};  // component subsampling (XRsiz, YRsiz)
    int cw[4] = {0, 0, 0, 0}, ch[4] = {0, 0, 0, 0};  // component sizes ceil(W/dx) x ceil(H/dy)
    size_t coff[5] = {0, 0, 0, 0, 0};                // element offset of each component's plane
    int roi[4] = {0, 0, 0, 0};                       // ROI maxshift per component (RGN; 0: none)
    std::vector<std::vector<Resolution>> geo;  // per component
    struct Job {
        int c, r, bi, i, j;  // component, resolution, band, block column, block row
    };
    std::vector<Job> jobs;
};
// One code-block coded with all passes (its codeword does not depend on
// Mb): the codeword's bytes (held by the caller), its passes and bit-planes.
struct CodedBlock {
    const uint8_t *data = nullptr;
    uint32_t len = 0;
    int passes = 0, numbps = 0;
    // Codeword segments (length, passes) when the style terminates passes
    // (BYPASS / TERMALL); none: one segment of len bytes.
    const std::pair<uint32_t, int> *seg = nullptr;
    int nseg = 0;
    // Bit-planes of the block's magnitudes before an ROI shift (-1: numbps).
    int numbps_plain = -1;
};
int encode_layout(const tc_encode_params &p, EncodeLayout &L, std::string &err);
// Guard bits from the blocks' bit-planes (unless p.guard_bits is set), Mb
// per band, zero bit-planes per block, packets and headers.
int encode_assemble(const tc_encode_params &p, EncodeLayout &L, const std::vector<CodedBlock> &coded,
                    std::vector<uint8_t> &out, std::string &err);
int encode_codestream(const tc_encode_params &p, const void *planes, std::vector<uint8_t> &out,
                      std::string &err);

}  // namespace tc
