// dwt_common.cuh -- helpers shared by the DWT kernels: whole-sample
// symmetric extension (ISO F.3.7) and the lifting constants and roundings.
#pragma once

#include "tc_j2k.h"

namespace tc {
namespace dwt {

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
