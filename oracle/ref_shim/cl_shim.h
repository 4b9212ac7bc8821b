/*
 * cl_shim.h -- lets the reference's OpenCL C kernels compile as host C/C++
 * (TEST INFRASTRUCTURE ONLY: builds oracle/_ref, the reference's own kernel
 * code run on the CPU, used to pin the oracle and as the CPU baseline).
 *
 * Work-item ids come from thread-local variables that the drivers in this
 * directory set before calling a kernel function once per work-item.  Only
 * kernels without work-group barriers are driven this way.
 */
#ifndef TC_CL_SHIM_H
#define TC_CL_SHIM_H

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

typedef unsigned int uint;
typedef unsigned char uchar;
typedef unsigned short ushort;
typedef struct { int x, y; } int2;

/* address-space and function qualifiers */
#define kernel
#define global
#define local
#ifdef __cplusplus
#define constant
#else
#define constant const
#endif

#ifdef __cplusplus
extern "C" {
#endif
extern __thread size_t shim_gid[3], shim_lid[3], shim_grp[3];
#ifdef __cplusplus
}
#endif

static inline size_t get_global_id(uint d) { return shim_gid[d]; }
static inline size_t get_local_id(uint d) { return shim_lid[d]; }
static inline size_t get_group_id(uint d) { return shim_grp[d]; }

#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
#ifdef SHIM_WORKGROUP_BARRIER
/* Kernels with work-group barriers: every work-item of a group runs on a
 * host thread of its own, and barrier() waits for the whole group (the
 * driver provides shim_group_barrier). */
void shim_group_barrier(void);
static inline void barrier(int flags) { (void)flags; shim_group_barrier(); }
#else
static inline void barrier(int flags) { (void)flags; }
#endif

static inline int clamp(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

/* round to nearest, ties to even, saturating (OpenCL convert_int_sat_rte) */
static inline int convert_int_sat_rte(float x)
{
    const double r = nearbyint((double)x);
    if (r >= 2147483647.0) return 2147483647;
    if (r <= -2147483648.0) return (-2147483647 - 1);
    return (int)r;
}

#endif
