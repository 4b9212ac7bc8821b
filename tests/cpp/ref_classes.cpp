// Drives the reference-named C++ classes of include/tc_j2k.hpp end to end:
// CoefficientCoder::decode_tile -> Quantizer::dequantize_tile -> DWT::iwt ->
// Preprocessor colour / DC shift, over a decode tree built from a descriptor
// file the test writes (one subband record per code-block, placed at the
// block's position in its component's Mallat plane).  The tree structs carry
// the field names of the reference's codestream_image_types.h, which the
// templates read.  Output: int32 samples, planar, to the output file.
//
// usage: ref_classes <input.bin> <output.bin>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "tc_j2k.hpp"

struct type_image;
struct type_tile;
struct type_subband;
typedef enum { LL, HL, LH, HH } type_orient;
struct type_codeblock {
    unsigned short tlx, tly, width, height;
    type_subband *parent_sb;
    unsigned char *codestream;
    unsigned int length;
    unsigned char significant_bits;
    unsigned int num_coding_passes;
    int d_coefficientsOffset;
};
struct type_subband {
    type_orient orient;
    unsigned short tlx, tly, width, height;
    unsigned int num_cblks;
    type_codeblock *cblks;
    unsigned char mag_bits;
    float step_size;
};
struct type_res_lvl {
    unsigned char num_subbands;
    type_subband *subbands;
};
struct type_tile_comp {
    unsigned short width, height;
    unsigned char num_dlvls, num_rlvls;
    void *img_data_d;
    type_res_lvl *res_lvls;
};
struct type_tile {
    void *coefficients;
    type_tile_comp *tile_comp;
    type_image *parent_img;
};
struct type_image {
    unsigned short width, height, num_components, depth;
    unsigned char sign, wavelet_type, use_mct;
    unsigned int num_tiles;
    type_tile *tile;
};

// input: int32 header [w, h, ncomp, bits, levels, reversible, mct, nblk, pool_len]
// then nblk records of int32 [comp, x, y, w, h, seg_off, seg_len, sigbits, passes, mb, orient] + float step
// then the pool bytes
int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int hd[9];
    if (std::fread(hd, 4, 9, f) != 9) return 2;
    const int W = hd[0], H = hd[1], C = hd[2], nblk = hd[7], pool_len = hd[8];
    std::vector<int> rec(11 * (size_t)nblk);
    std::vector<float> steps(nblk);
    for (int i = 0; i < nblk; i++)
        if (std::fread(&rec[11 * (size_t)i], 4, 11, f) != 11 || std::fread(&steps[i], 4, 1, f) != 1) return 2;
    std::vector<unsigned char> pool(pool_len + 16);
    if (std::fread(pool.data(), 1, pool_len, f) != (size_t)pool_len) return 2;
    std::fclose(f);

    type_image img{};
    img.width = W;
    img.height = H;
    img.num_components = C;
    img.depth = hd[3];
    img.wavelet_type = hd[5] ? 0 : 1;
    img.use_mct = hd[6];
    img.num_tiles = 1;
    type_tile tile{};
    std::vector<type_tile_comp> comps(C);
    std::vector<std::vector<type_subband>> sbs(C);
    std::vector<type_codeblock> cbs(nblk);
    for (int i = 0; i < nblk; i++) sbs[rec[11 * (size_t)i]].push_back(type_subband{});
    std::vector<int> fill(C, 0);
    for (int i = 0; i < nblk; i++) {
        const int *r = &rec[11 * (size_t)i];
        type_subband &sb = sbs[r[0]][fill[r[0]]++];
        type_codeblock &cb = cbs[i];
        sb.orient = (type_orient)r[10];
        sb.tlx = r[1];
        sb.tly = r[2];
        sb.width = r[3];
        sb.height = r[4];
        sb.num_cblks = 1;
        sb.cblks = &cb;
        sb.mag_bits = r[9];
        sb.step_size = steps[i];
        cb.width = r[3];
        cb.height = r[4];
        cb.parent_sb = &sb;
        cb.codestream = pool.data() + r[5];
        cb.length = r[6];
        cb.significant_bits = r[7];
        cb.num_coding_passes = r[8];
    }
    for (int c = 0; c < C; c++) {
        comps[c].width = W;
        comps[c].height = H;
        comps[c].num_dlvls = hd[4];
    }
    // a resolution level may hold more subbands than an unsigned char counts:
    // split each component's records over as many levels as needed
    std::vector<std::vector<type_res_lvl>> many(C);
    for (int c = 0; c < C; c++) {
        for (size_t k = 0; k < sbs[c].size(); k += 255) {
            type_res_lvl rl{};
            rl.num_subbands = (unsigned char)std::min<size_t>(255, sbs[c].size() - k);
            rl.subbands = &sbs[c][k];
            many[c].push_back(rl);
        }
        comps[c].num_rlvls = (unsigned char)many[c].size();
        comps[c].res_lvls = many[c].data();
    }
    tile.tile_comp = comps.data();
    tile.parent_img = &img;
    img.tile = &tile;

    try {
        tc::Context ctx(0);
        tc::CoefficientCoder coder(ctx.get());
        tc::Quantizer quant(ctx.get());
        tc::DWT dwt(ctx.get());
        tc::Preprocessor pre(ctx.get());
        coder.decode_tile(&tile);
        quant.dequantize_tile(&tile);
        dwt.iwt(&tile);
        if (img.use_mct && C >= 3) {
            if (img.wavelet_type ? pre.color_decoder_lossy(&img) : pre.color_decoder_lossless(&img)) return 3;
        } else {
            pre.idc_level_shifting(&img);
        }
        std::vector<int> out((size_t)W * H * C);
        for (int c = 0; c < C; c++)
            tc::check_cuda(cudaMemcpy(out.data() + (size_t)c * W * H, comps[c].img_data_d, (size_t)W * H * 4,
                                      cudaMemcpyDeviceToHost), "read back");
        FILE *o = std::fopen(argv[2], "wb");
        if (!o) return 2;
        std::fwrite(out.data(), 4, out.size(), o);
        std::fclose(o);
    } catch (const tc::Error &e) {
        std::fprintf(stderr, "tc::Error %d: %s\n", e.status(), e.what());
        return 4;
    }
    return 0;
}
