// dwt_common.cuh -- helpers shared by the DWT kernels: whole-sample
// symmetric extension (ISO F.3.7) and the lifting constants and roundings.
#pragma once

#include <cuda_runtime.h>

#include "tc_j2k.h"

namespace tc {
namespace dwt {

// Programmatic dependent launch between the reverse levels: a level's grid
// lets the next level's grid be scheduled once all its CTAs have started
// (launch_dependents), and a level waits for the previous one to complete
// and flush before it reads that level's output (wait).  Without a
// programmatic predecessor the wait returns at once.
__device__ __forceinline__ void pdl_allow_next() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait_prev() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Launches kernel<<<grid, block, smem, stream>>>(args...) with programmatic
// stream serialisation allowed, so its CTAs may be scheduled while the
// previous kernel on the stream finishes (the kernel must pdl_wait_prev()
// before it reads what that kernel wrote).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

__device__ __forceinline__ int pse(int i, int n)
{
    if (n == 1) return 0;
    const int per = 2 * (n - 1);
    i %= per;
    if (i < 0) i += per;
    return i >= n ? per - i : i;
}

// Index inside [0, n) after extension; the modulo path only runs at borders.
__device__ __forceinline__ int mirror(int i, int n)
{
    return (unsigned)i < (unsigned)n ? i : pse(i, n);
}

// 9/7 lifting constants (ISO F.4.8.2).
constexpr float kA = -1.586134342059924f, kB = -0.052980118572961f, kG = 0.882911075530934f,
                kD = 0.443506852043971f, kK = 1.230174104914001f, kInvK = 1.0f / 1.230174104914001f;
// Scaling-free reverse lifting: with E = X(2n)/K and O = X(2n+1)*K lifted in
// place of the K-scaled samples of ISO F.3.8.2, the four steps become
// E -= (delta/K^2)(O + O'), O -= (gamma K^2)(E + E'), E -= (beta/K^2)(..),
// O -= (alpha K^2)(..), and a row-then-column level leaves each output off
// by a factor of K^2 (even row and column), 1/K^2 (odd, odd) or 1.
constexpr double kK2d = 1.230174104914001 * 1.230174104914001;
constexpr float kSfD = (float)(0.443506852043971 / kK2d), kSfG = (float)(0.882911075530934 * kK2d),
                kSfB = (float)(-0.052980118572961 / kK2d), kSfA = (float)(-1.586134342059924 * kK2d),
                kSfEven = (float)kK2d, kSfOdd = (float)(1.0 / kK2d);

// Combined output factor of the scaling-free row and column passes of a
// 9/7 level, by the parity of the output row and column: K^2, 1, 1, 1/K^2
// (a pass that did not run, over a single row or column, contributes 1).
__device__ __forceinline__ float sf_factor(int row_odd, int col_odd, bool rows_lifted, bool cols_lifted)
{
    const float fc = rows_lifted ? (col_odd ? kInvK : kK) : 1.0f;
    const float fr = cols_lifted ? (row_odd ? kInvK : kK) : 1.0f;
    if (rows_lifted && cols_lifted) return row_odd == col_odd ? (row_odd ? kSfOdd : kSfEven) : 1.0f;
    return fc * fr;
}

template <int RND>
__device__ __forceinline__ int div4r(int v)
{
    return RND == TC_ROUND_TRUNC ? v / 4 : (v >> 2);
}
template <int RND>
__device__ __forceinline__ int div2r(int v)
{
    return RND == TC_ROUND_TRUNC ? v / 2 : (v >> 1);
}

}  // namespace dwt
}  // namespace tc
