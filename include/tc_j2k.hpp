/*
 * tc_j2k.hpp -- the reference's stage classes, header-only, over tc_j2k.h.
 *
 * kgmoore/ThousandthChicken's host code drives its device stages through
 * C++ classes: CoefficientCoder (CoefficientCoder.h:37-48), Quantizer
 * (Quantizer.h:9-17), DWTKernel<T> with DWTForward53/97 and DWTReverse53/97
 * (DWTKernel.h:11-13), DWT (DWT.h:14-18), Preprocessor (Preprocessor.h:22-24)
 * and Decoder (Decoder.h:18-20).  This header gives a C++ caller of that code
 * the same names and call shapes, so the calls stay as they are and only the
 * construction changes: each class takes a tc_ctx (a CUDA device and stream)
 * where the reference took KernelInitInfoBase{cmd_queue, buildOptions}.
 *
 * The tile walkers are templates over the reference's decode tree
 * (type_tile / type_tile_comp / type_res_lvl / type_subband /
 * type_codeblock / type_image, codestream_image_types.h:30-424): they use
 * those structs' field names and need no declaration from this header, so
 * the header compiles with or without the reference's headers.
 *
 * Differences a caller sees:
 *  - errors throw tc::Error (status and message) where the reference threw
 *    Error from SAMPLE_CHECK_ERRORS (basic.h:95-104);
 *  - device buffers are CUDA device pointers (void *) where the reference
 *    had cl_mem (platform.h:9-11);
 *  - CoefficientCoder::decode_tile writes raw sign-magnitude words straight
 *    at each block's place in the tile component's Mallat plane, and
 *    cblk->d_coefficientsOffset holds that element offset (the reference
 *    used one nominal-size slot per block, CoefficientCoder.cpp:129);
 *    Quantizer::dequantize_tile turns them into values in img_data_d;
 *  - a block whose num_coding_passes is 0 while it has codeword bytes is
 *    decoded with every pass of its significant bit-planes: the reference's
 *    parser never fills the count (defect D3) and its kernel decodes them
 *    all;
 *  - DWT::iwt frees the plane it replaces when this header allocated it (the
 *    reference leaks it, DWT.cpp:79-96).
 */
#ifndef TC_J2K_HPP
#define TC_J2K_HPP

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "tc_j2k.h"

namespace tc {

class Error : public std::runtime_error {
public:
    Error(int status, const std::string &what) : std::runtime_error(what), status_(status) {}
    int status() const { return status_; }

private:
    int status_;
};

inline void check(int status, tc_ctx *ctx, const char *what)
{
    if (status == TC_OK) return;
    std::string m = std::string(what) + ": " + tc_status_string(status);
    if (ctx && *tc_ctx_last_error(ctx)) m += std::string(" (") + tc_ctx_last_error(ctx) + ")";
    throw Error(status, m);
}

inline void check_cuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw Error(TC_E_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}

/* A device buffer the classes own (freed with them). */
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    DeviceBuffer(DeviceBuffer &&o) noexcept : ptr_(o.ptr_), size_(o.size_) { o.ptr_ = nullptr, o.size_ = 0; }
    DeviceBuffer &operator=(DeviceBuffer &&o) noexcept
    {
        if (this != &o) {
            release();
            ptr_ = o.ptr_;
            size_ = o.size_;
            o.ptr_ = nullptr;
            o.size_ = 0;
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void *ensure(size_t bytes)
    {
        if (bytes > size_) {
            release();
            check_cuda(cudaMalloc(&ptr_, bytes ? bytes : 16), "cudaMalloc");
            size_ = bytes;
        }
        return ptr_;
    }
    void release()
    {
        if (ptr_) cudaFree(ptr_);
        ptr_ = nullptr;
        size_ = 0;
    }
    void *get() const { return ptr_; }

private:
    void *ptr_ = nullptr;
    size_t size_ = 0;
};

/* Owns a tc_ctx: the device and stream every class below works on
 * (replaces InitOpenCL and KernelInitInfoBase, ocl_util.cpp:425-466,
 * platform.h:21-34). */
class Context {
public:
    explicit Context(int device = 0, cudaStream_t stream = nullptr)
    {
        check(tc_ctx_create(device, stream, &ctx_), nullptr, "tc_ctx_create");
    }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    ~Context()
    {
        if (ctx_) tc_ctx_destroy(ctx_);
    }
    tc_ctx *get() const { return ctx_; }
    void synchronize() { check(tc_ctx_synchronize(ctx_), ctx_, "tc_ctx_synchronize"); }

private:
    tc_ctx *ctx_ = nullptr;
};

namespace detail {

/* The code-blocks of a tile as descriptors over a host segment pool, placed
 * in each tile component's Mallat plane (subband sb->tlx/tly plus block
 * cblk->tlx/tly, pitch tile_comp->width; codestream_image.c:96-108), the
 * components' planes one after another.  comp_off[c] receives component c's
 * first element. */
template <class Tile>
void tile_blocks(Tile *tile, std::vector<tc_cblk_desc> &desc, std::vector<uint8_t> *pool,
                 std::vector<uint64_t> &comp_off, bool set_offsets)
{
    auto *img = tile->parent_img;
    const bool irrev = img->wavelet_type != 0;
    uint64_t base = 0;
    desc.clear();
    comp_off.clear();
    for (int c = 0; c < (int)img->num_components; c++) {
        auto *tc = &tile->tile_comp[c];
        comp_off.push_back(base);
        for (int r = 0; r < (int)tc->num_rlvls; r++) {
            auto *rl = &tc->res_lvls[r];
            for (int s = 0; s < (int)rl->num_subbands; s++) {
                auto *sb = &rl->subbands[s];
                for (unsigned k = 0; k < sb->num_cblks; k++) {
                    auto *cb = &sb->cblks[k];
                    tc_cblk_desc d;
                    std::memset(&d, 0, sizeof d);
                    if (pool) {
                        d.seg_off = pool->size();
                        if (cb->length) pool->insert(pool->end(), cb->codestream, cb->codestream + cb->length);
                        pool->resize((pool->size() + 15) & ~size_t(15));
                    }
                    d.seg_len = cb->length;
                    d.out_off = base + (uint64_t)(sb->tly + cb->tly) * tc->width + sb->tlx + cb->tlx;
                    d.out_pitch = tc->width;
                    d.w = cb->width;
                    d.h = cb->height;
                    const int sig = cb->significant_bits;
                    int passes = (int)cb->num_coding_passes;
                    if (passes == 0 && cb->length > 0 && sig > 0) passes = 3 * sig - 2;   // D3
                    d.passes = (uint8_t)passes;
                    d.mb = sb->mag_bits;
                    d.zero_bitplanes = (uint8_t)(sb->mag_bits > sig ? sb->mag_bits - sig : 0);
                    d.orient = (uint8_t)sb->orient;
                    d.step = irrev ? (float)sb->step_size : 1.0f;
                    d.flags = irrev ? TC_CBLK_IRREVERSIBLE : 0;
                    if (set_offsets) cb->d_coefficientsOffset = (int)d.out_off;
                    desc.push_back(d);
                }
            }
        }
        base += (uint64_t)tc->width * tc->height;
    }
    comp_off.push_back(base);
}

}  // namespace detail

/* CoefficientCoder (CoefficientCoder.h:37-48, CoefficientCoder.cpp:62-252). */
class CoefficientCoder {
public:
    explicit CoefficientCoder(tc_ctx *ctx) : ctx_(ctx) {}

    /* Tier-1 of every code-block of the tile in one persistent launch,
     * longest blocks first: raw sign-magnitude words (the reference's
     * g_decode output, coefficient_coder.cl:605-626) at each block's place
     * in tile->coefficients, a device arena this object owns. */
    template <class Tile>
    void decode_tile(Tile *tile)
    {
        std::vector<tc_cblk_desc> desc;
        std::vector<uint8_t> pool;
        std::vector<uint64_t> comp_off;
        detail::tile_blocks(tile, desc, &pool, comp_off, true);
        const uint64_t elems = comp_off.back();
        std::vector<uint32_t> order(desc.size());
        check(tc_t1_sort_order(desc.data(), (int)desc.size(), order.data()), ctx_, "tc_t1_sort_order");
        cudaStream_t st = static_cast<cudaStream_t>(tc_ctx_stream(ctx_));
        void *d_pool = pool_.ensure(pool.size() + 16);
        void *d_desc = desc_.ensure(desc.size() * sizeof(tc_cblk_desc) + 16);
        void *d_order = order_.ensure(order.size() * 4 + 16);
        void *d_coef = coef_.ensure(elems * 4 + 16);
        check_cuda(cudaMemcpyAsync(d_pool, pool.data(), pool.size(), cudaMemcpyHostToDevice, st), "upload");
        check_cuda(cudaMemcpyAsync(d_desc, desc.data(), desc.size() * sizeof(tc_cblk_desc), cudaMemcpyHostToDevice,
                                   st), "upload");
        check_cuda(cudaMemcpyAsync(d_order, order.data(), order.size() * 4, cudaMemcpyHostToDevice, st), "upload");
        check_cuda(cudaMemsetAsync(d_coef, 0, elems * 4, st), "clear");
        check(tc_t1_decode(ctx_, static_cast<tc_cblk_desc *>(d_desc), static_cast<uint32_t *>(d_order),
                           (int)desc.size(), static_cast<uint8_t *>(d_pool), pool.size(), d_coef, elems,
                           TC_T1_OUT_RAW, 0.0f, 31),
              ctx_, "tc_t1_decode");
        check(tc_ctx_synchronize(ctx_), ctx_, "tc_t1_decode");
        tile->coefficients = d_coef;
    }

private:
    tc_ctx *ctx_;
    DeviceBuffer pool_, desc_, order_, coef_;
};

/* Quantizer (Quantizer.h:9-17, Quantizer.cpp:181-216): the raw words of
 * tile->coefficients to int32 (5/3) or float (9/7) values in each tile
 * component's img_data_d, a plane this object owns.  recon_r is the
 * reconstruction point of ISO E.1.1.2 (0 = the truncated value). */
class Quantizer {
public:
    explicit Quantizer(tc_ctx *ctx, float recon_r = 0.5f) : ctx_(ctx), r_(recon_r) {}

    template <class Tile>
    void dequantize_tile(Tile *tile)
    {
        std::vector<tc_cblk_desc> desc;
        std::vector<uint64_t> comp_off;
        detail::tile_blocks(tile, desc, nullptr, comp_off, false);
        const uint64_t elems = comp_off.back();
        void *d_desc = desc_.ensure(desc.size() * sizeof(tc_cblk_desc) + 16);
        char *d_out = static_cast<char *>(out_.ensure(elems * 4 + 16));
        cudaStream_t st = static_cast<cudaStream_t>(tc_ctx_stream(ctx_));
        check_cuda(cudaMemcpyAsync(d_desc, desc.data(), desc.size() * sizeof(tc_cblk_desc), cudaMemcpyHostToDevice,
                                   st), "upload");
        check_cuda(cudaMemsetAsync(d_out, 0, elems * 4, st), "clear");
        check(tc_dequantize_raw(ctx_, static_cast<tc_cblk_desc *>(d_desc), (int)desc.size(),
                                static_cast<const uint32_t *>(tile->coefficients), d_out, elems, r_),
              ctx_, "tc_dequantize_raw");
        check(tc_ctx_synchronize(ctx_), ctx_, "tc_dequantize_raw");
        for (int c = 0; c < (int)tile->parent_img->num_components; c++)
            tile->tile_comp[c].img_data_d = d_out + comp_off[c] * 4;
    }

private:
    tc_ctx *ctx_;
    float r_;
    DeviceBuffer desc_, out_;
};

/* DWTKernel<T>::run(in, out, sizeX, sizeY, levels) (DWTKernel.h:11-13,
 * DWTKernel.cpp:158-178) with DWTForward53/97 and DWTReverse53/97: T is
 * int (5/3) or float (9/7); planes of sizeX x sizeY, pitch sizeX, Mallat
 * layout on the transformed side. */
template <typename T>
class DWTKernel {
public:
    explicit DWTKernel(tc_ctx *ctx) : ctx_(ctx) {}
    virtual ~DWTKernel() = default;
    int run(void *in, void *out, int sizeX, int sizeY, int levels)
    {
        const int rc = dwt(in, out, sizeX, sizeY, levels);
        check(rc, ctx_, "DWTKernel::run");
        return rc;
    }

protected:
    virtual int dwt(void *in, void *out, int sx, int sy, int levels) = 0;
    tc_ctx *ctx_;
};

class DWTForward53 : public DWTKernel<int> {
public:
    using DWTKernel<int>::DWTKernel;

protected:
    int dwt(void *in, void *out, int sx, int sy, int levels) override
    {
        return tc_dwt_forward53(ctx_, static_cast<const int32_t *>(in), sx, static_cast<int32_t *>(out), sx, sx, sy,
                                levels, TC_ROUND_FLOOR);
    }
};

class DWTReverse53 : public DWTKernel<int> {
public:
    using DWTKernel<int>::DWTKernel;

protected:
    int dwt(void *in, void *out, int sx, int sy, int levels) override
    {
        return tc_dwt_reverse53(ctx_, static_cast<const int32_t *>(in), sx, static_cast<int32_t *>(out), sx, sx, sy,
                                levels, TC_ROUND_FLOOR);
    }
};

class DWTForward97 : public DWTKernel<float> {
public:
    using DWTKernel<float>::DWTKernel;

protected:
    int dwt(void *in, void *out, int sx, int sy, int levels) override
    {
        return tc_dwt_forward97(ctx_, static_cast<const float *>(in), sx, static_cast<float *>(out), sx, sx, sy,
                                levels);
    }
};

class DWTReverse97 : public DWTKernel<float> {
public:
    using DWTKernel<float>::DWTKernel;

protected:
    int dwt(void *in, void *out, int sx, int sy, int levels) override
    {
        return tc_dwt_reverse97(ctx_, static_cast<const float *>(in), sx, static_cast<float *>(out), sx, sx, sy,
                                levels);
    }
};

/* DWT::iwt (DWT.h:14-18, DWT.cpp:57-114): the reverse transform of every
 * tile component, whose img_data_d then points at the transformed plane
 * (owned by this object). */
class DWT {
public:
    explicit DWT(tc_ctx *ctx) : ctx_(ctx), r53_(ctx), r97_(ctx) {}

    template <class Tile>
    void iwt(Tile *tile)
    {
        auto *img = tile->parent_img;
        planes_.resize(img->num_components);
        for (int c = 0; c < (int)img->num_components; c++) {
            auto *tc = &tile->tile_comp[c];
            void *out = planes_[c].ensure((size_t)tc->width * tc->height * 4 + 16);
            if (img->wavelet_type) r97_.run(tc->img_data_d, out, tc->width, tc->height, tc->num_dlvls);
            else r53_.run(tc->img_data_d, out, tc->width, tc->height, tc->num_dlvls);
            tc->img_data_d = out;
        }
        check(tc_ctx_synchronize(ctx_), ctx_, "DWT::iwt");
    }

private:
    tc_ctx *ctx_;
    DWTReverse53 r53_;
    DWTReverse97 r97_;
    std::vector<DeviceBuffer> planes_;
};

/* Preprocessor (Preprocessor.h:22-24, Preprocessor.cpp:44-306): inverse
 * colour transforms and DC level shift on every tile's components, in place
 * on their img_data_d planes, int32 samples out (clamped to the image's
 * depth).  The colour transforms return -1 for images of fewer than three
 * components, as the reference does. */
class Preprocessor {
public:
    explicit Preprocessor(tc_ctx *ctx) : ctx_(ctx) {}

    template <class Image>
    int color_decoder_lossless(Image *img)
    {
        return color(img, TC_COLOR_RCT);
    }
    template <class Image>
    int color_decoder_lossy(Image *img)
    {
        return color(img, TC_COLOR_ICT);
    }
    template <class Image>
    void idc_level_shifting(Image *img)
    {
        for (unsigned t = 0; t < img->num_tiles; t++)
            for (int c = 0; c < (int)img->num_components; c++) one(img, &img->tile[t], c, 1, TC_COLOR_DC);
        check(tc_ctx_synchronize(ctx_), ctx_, "Preprocessor");
    }

private:
    template <class Image>
    int color(Image *img, int kind)
    {
        if (img->num_components < 3) return -1;
        for (unsigned t = 0; t < img->num_tiles; t++) {
            one(img, &img->tile[t], 0, 3, kind);
            for (int c = 3; c < (int)img->num_components; c++) one(img, &img->tile[t], c, 1, TC_COLOR_DC);
        }
        check(tc_ctx_synchronize(ctx_), ctx_, "Preprocessor");
        return 0;
    }
    template <class Image, class Tile>
    void one(Image *img, Tile *tile, int c0, int n, int kind)
    {
        void *planes[4] = {nullptr, nullptr, nullptr, nullptr};
        for (int k = 0; k < n; k++) planes[k] = tile->tile_comp[c0 + k].img_data_d;
        auto *tc = &tile->tile_comp[c0];
        const int bits = img->depth | (img->sign ? TC_SIGNED : 0);
        check(tc_color_inverse(ctx_, kind, n, planes, img->wavelet_type ? TC_FLOAT32 : TC_INT32, tc->width, planes,
                               TC_INT32, tc->width, tc->width, tc->height, bits),
              ctx_, "tc_color_inverse");
    }
    tc_ctx *ctx_;
};

/* Decoder (Decoder.h:14-33, Decoder.cpp:94-217): a whole codestream or JP2
 * file to planar host samples (8-bit when the depth is at most 8, else
 * 16-bit).  decode returns 0, or -2 when the file is missing
 * (Decoder.cpp:103-107); other failures throw. */
class Decoder {
public:
    explicit Decoder(tc_ctx *ctx) : ctx_(ctx) {}
    int decode(const std::string &fileName)
    {
        tc_image_info info;
        std::vector<uint8_t> out;
        const int rc = decode(fileName, out, info);
        return rc == TC_E_NOFILE ? -2 : 0;
    }
    int decode(const std::string &fileName, std::vector<uint8_t> &out, tc_image_info &info)
    {
        FILE *f = std::fopen(fileName.c_str(), "rb");
        if (!f) return TC_E_NOFILE;
        std::vector<uint8_t> cs;
        uint8_t buf[1 << 16];
        size_t n;
        while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) cs.insert(cs.end(), buf, buf + n);
        std::fclose(f);
        check(tc_j2k_read_header(cs.data(), cs.size(), &info), ctx_, "tc_j2k_read_header");
        size_t bytes = 0;
        for (int c = 0; c < info.ncomp; c++) {
            const int dx = info.comp_dx[c] ? info.comp_dx[c] : 1, dy = info.comp_dy[c] ? info.comp_dy[c] : 1;
            bytes += (size_t)((info.width + dx - 1) / dx) * ((info.height + dy - 1) / dy);
        }
        bytes *= info.bits <= 8 ? 1 : 2;
        out.resize(bytes);
        check(tc_decode_j2k(ctx_, cs.data(), cs.size(), out.data(), out.size(), &info), ctx_, "tc_decode_j2k");
        return TC_OK;
    }

private:
    tc_ctx *ctx_;
};

}  // namespace tc

#endif /* TC_J2K_HPP */
