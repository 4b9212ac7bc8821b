/*
 * ref_dwt53.cc -- host driver for the reference's 5/3 DWT kernels
 * (dwt_f53.cl or dwt_r53.cl, chosen by REF_DWT53_FORWARD), compiled from the
 * reference source with cl_shim.h.  TEST INFRASTRUCTURE ONLY.
 *
 * The kernels synchronise the work-items of a group through local memory
 * (localMemoryFence, platform.cl), so each group runs as WIN_SIZE_X host
 * threads sharing the group's local buffer and a std::barrier.  Each
 * work-item keeps its own copy of the kernel-scope TransformBufferINT: it
 * holds only sizes, the same for every work-item, and the pointer to the
 * shared local buffer.  One level is enqueued as DWTKernel<T>::enqueue does
 * (DWTKernel.cpp:88-124): the window by image width as DWTForward53::dwt /
 * DWTReverse53::dwt choose it (192, 128 or 64 columns by 8 rows), the
 * sliding-window step count divRndUp(sy, 15 * WIN_SY), and the local buffer
 * size of calcTransformDataBufferSize (DWTKernel.cpp:193-201).  The
 * multi-level recursion with copyLLBandToSrc runs in the caller.
 *
 * OpenCL local memory starts undefined; here every group's buffer starts
 * filled with REF_DWT53_FILL (default 0).  At image widths that are not a
 * multiple of the window the kernels read cells no work-item wrote, and
 * their output changes with the fill; at window-multiple widths it does not
 * (the tests compare only those).
 */
// the standard headers first: the shim's address-space macros (local,
// global, kernel) would break them
#include <algorithm>
#include <barrier>
#include <cstdlib>
#include <thread>
#include <vector>

#define SHIM_WORKGROUP_BARRIER 1
#include "cl_shim.h"

#ifdef REF_DWT53_FORWARD
#include "dwt_f53.cl"
#else
#include "dwt_r53.cl"
#endif

__thread size_t shim_gid[3], shim_lid[3], shim_grp[3];
static thread_local std::barrier<> *g_group_barrier = nullptr;

void shim_group_barrier(void) { g_group_barrier->arrive_and_wait(); }

static int div_up(int n, int d) { return n / d + !!(n % d); }

/* One level of the 5/3 transform of an sx x sy image in the reference's
 * band layout: in and out hold sx * sy int32 (in is read, out written).
 * Returns the number of work-groups run. */
extern "C" int REF_DWT53_NAME(const int *in, int *out, int sx, int sy)
{
    const int WX = sx >= 960 ? 192 : (sx >= 480 ? 128 : 64), WY = 8;
    const int diameter = 3;   // DWTForward53 / DWTReverse53 construct DWTKernel<int>(3, ...)
    const int wsy = WY + diameter, bx = (diameter + 1) / 2, stride = bx + WX / 2;
    const int bsize = stride * wsy, pad = 32 - ((bsize + 16) % 32);
    const int local_ints = 2 * bsize + pad;
    const int steps = div_up(sy, 15 * WY);
    const int gx = div_up(sx, WX), gy = div_up(sy, WY * steps);
    std::vector<int> data((size_t)local_ints);
    const int fill = getenv("REF_DWT53_FILL") ? atoi(getenv("REF_DWT53_FILL")) : 0;
    for (int g1 = 0; g1 < gy; g1++)
        for (int g0 = 0; g0 < gx; g0++) {
            std::fill(data.begin(), data.end(), fill);
            std::barrier<> bar(WX);
            std::vector<std::thread> items;
            items.reserve(WX);
            for (int l = 0; l < WX; l++)
                items.emplace_back([&, l] {
                    g_group_barrier = &bar;
                    shim_grp[0] = (size_t)g0;
                    shim_grp[1] = (size_t)g1;
                    shim_grp[2] = 0;
                    shim_lid[0] = (size_t)l;
                    shim_lid[1] = shim_lid[2] = 0;
                    shim_gid[0] = (size_t)g0 * WX + l;
                    shim_gid[1] = (size_t)g1;
                    shim_gid[2] = 0;
                    run(WX, WY, data.data(), in, out, sx, sy, steps);
                });
            for (std::thread &t : items) t.join();
        }
    return gx * gy;
}
