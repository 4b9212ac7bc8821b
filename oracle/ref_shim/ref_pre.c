/*
 * ref_pre.c -- host drivers for the reference's colour / DC-shift kernels
 * (preprocess_*.cl) and dequantiser kernels (quantizer_*_inverse.cl),
 * compiled from the reference sources with cl_shim.h.  TEST INFRASTRUCTURE
 * ONLY.  One call of the kernel function per work-item.
 */
#include "cl_shim.h"
#include "preprocess_rct.cl"
#include "preprocess_rct_inverse.cl"
#include "preprocess_ict.cl"
#include "preprocess_ict_inverse.cl"
#include "preprocess_dc_level_shift.cl"
#include "preprocess_dc_level_shift_inverse.cl"
#include "quantizer_lossless_inverse.cl"
#include "quantizer_lossy_inverse.cl"

__thread size_t shim_gid[3], shim_lid[3], shim_grp[3];

#define EACH(n) for (size_t i_ = 0; i_ < (size_t)(n); i_++) if ((shim_gid[0] = i_), 1)

void ref_rct(int *r, int *g, int *b, int n, int level_shift) { EACH(n) rct_kernel(r, g, b, 0, 0, level_shift); }
void ref_rct_inverse(int *y, int *u, int *v, int n, int level_shift, int mn, int mx)
{
    EACH(n) tcr_kernel(y, u, v, 0, 0, level_shift, mn, mx);
}
void ref_ict(int *r, int *g, int *b, int n, int level_shift) { EACH(n) ict_kernel(r, g, b, 0, 0, level_shift); }
void ref_ict_inverse(int *y, int *u, int *v, int n, int level_shift, int mn, int mx)
{
    EACH(n) tci_kernel(y, u, v, 0, 0, level_shift, mn, mx);
}
void ref_dc_shift(int *x, int n, int level_shift) { EACH(n) fdc_level_shift_kernel(x, 0, 0, level_shift); }
void ref_dc_shift_inverse(int *x, int n, int level_shift, int mn, int mx)
{
    EACH(n) idc_level_shift_kernel(x, 0, 0, level_shift, mn, mx);
}

/* One code-block of w x h words at in (pitch in_pitch) -> out (pitch
 * out_pitch), one 16x16 work-group as Quantizer::dequantization launches it
 * per block (Quantizer.cpp:160-171). */
static void run_group(int lossy, int *in, int in_pitch, int *out, int out_pitch, int w, int h, int shift,
                      float factor)
{
    int2 isize = {in_pitch, h}, osize = {out_pitch, h}, cb = {w, h};
    shim_grp[0] = shim_grp[1] = 0;
    for (int ly = 0; ly < BLOCKSIZEY; ly++)
        for (int lx = 0; lx < BLOCKSIZEX; lx++) {
            shim_lid[0] = (size_t)lx;
            shim_lid[1] = (size_t)ly;
            if (lossy) subband_dequantization_lossy(in, isize, out, 0, osize, cb, factor);
            else subband_dequantization_lossless(in, isize, out, 0, osize, cb, shift);
        }
}

void ref_dequant_lossless(int *in, int *out, int w, int h, int shift) { run_group(0, in, w, out, w, w, h, shift, 0.f); }
void ref_dequant_lossy(int *in, int *out, int w, int h, float f) { run_group(1, in, w, out, w, w, h, 0, f); }
