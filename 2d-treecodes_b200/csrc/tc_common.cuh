// tc_common.cuh -- shared constants, error plumbing and device helpers of the B200 treecode.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "treecodes_b200.h"

namespace tc {

// Compile-time parameters of the reference build (Makefile:13-15 of the reference,
// drivers/Makefile:20): expansion order 12 for the potential, 24 for the force, MRAG block
// of 32 x 32 targets, deepest level 15, leaf capacities 512 / 192
// (drivers/treecode-potential.cpp:99, drivers/treecode-force.cpp:216), bricks of 8 x 8
// (drivers/treecode-force.cpp:91).
constexpr int LMAX = 15;
constexpr int BLOCKSIZE = 32;
constexpr int TILE = 8;
constexpr int ORDER_POTENTIAL = 12;
constexpr int ORDER_FORCE = 24;
constexpr int LEAF_POTENTIAL = 32 * 16;
constexpr int LEAF_FORCE = 192;
constexpr int MAX_ORDER = 32;

// Status codes: tc_status of the C ABI (treecodes_b200.h).

// Device-side error word bits (set by kernels, read by the host after the call).
enum DeviceError : unsigned {
    DEVERR_SPIN_LIMIT = 1u << 0,   // a bounded wait gave up
    DEVERR_STACK = 1u << 1,        // traversal stack overflow
    DEVERR_TREE = 1u << 2,         // inconsistent tree bookkeeping
    DEVERR_BOUNDS = 1u << 3,       // an index failed its bounds check (access skipped)
};

// Coordinate frame of a source set: sort-sources.cpp:78-82 of the reference.
struct Frame {
    double xmin, ymin, ext;   // padded bounding square
    double scale;             // (1 / ext) * 2^LMAX, the factor the compiled reference uses
};

constexpr unsigned FULL_MASK = 0xffffffffu;

// Reads without progress after which a device wait on another CTA's published state gives up
// and raises DEVERR_SPIN_LIMIT (a context's test setting can lower it, tc_set_wait_test).
constexpr int DEFAULT_SPIN_LIMIT = 1 << 22;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Programmatic dependent launch (launch_pdl): a kernel may be scheduled while the kernel before
// it on its stream is still draining.  A kernel so launched calls this first: it waits until
// that kernel has completed and its writes are visible (so stream order holds exactly), then
// lets the kernel after it be scheduled in turn.  Both are no-ops without the launch attribute.
__device__ __forceinline__ void pdl_begin() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Approximate FP64 reciprocal from the SFU (PTX rcp.approx.ftz.f64), refined by two
// Newton-Raphson steps y <- y + y (1 - d y); each step doubles the number of correct bits.
__device__ __forceinline__ double rcp_nr(double d) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    double e = fma(-d, y, 1.0);
    y = fma(y, e, y);
    e = fma(-d, y, 1.0);
    y = fma(y, e, y);
    return y;
}

__device__ __forceinline__ double shfl_xor_d(double v, int m) {
    return __shfl_xor_sync(FULL_MASK, v, m);
}

// Morton interleave of a 15-bit coordinate: sort-sources.cpp:96-104 of the reference.
__host__ __device__ __forceinline__ int spread_bits(int x) {
    x = (x | (x << 8)) & 0x00FF00FF;
    x = (x | (x << 4)) & 0x0F0F0F0F;
    x = (x | (x << 2)) & 0x33333333;
    x = (x | (x << 1)) & 0x55555555;
    return x;
}

__host__ __device__ __forceinline__ int compact_bits(int x) {
    x &= 0x55555555;
    x = (x | (x >> 1)) & 0x33333333;
    x = (x | (x >> 2)) & 0x0F0F0F0F;
    x = (x | (x >> 4)) & 0x00FF00FF;
    x = (x | (x >> 8)) & 0x0000FFFF;
    return x;
}

// Node record read by the traversals: centre of mass, radius, first child (-1: leaf) and the
// number of sources the node hands to P2P (0 for empty leaves).
struct __align__(32) TNode {
    double xcom, ycom, r;
    int child;
    int count;
};

// Block-wide exclusive scan of one int per thread (blockDim.x a multiple of 32, <= 1024); the
// block total goes to *total when total is not null.  Every thread of the block must call it.
__device__ __forceinline__ int block_exclusive_scan(int v, int *total) {
    __shared__ int warp_sums[32];
    const int lane = lane_id(), w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULL_MASK, inc, o);
        if (lane >= o) inc += t;
    }
    __syncthreads();
    if (lane == 31) warp_sums[w] = inc;
    __syncthreads();
    if (w == 0) {
        int s = lane < nw ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(FULL_MASK, s, o);
            if (lane >= o) s += t;
        }
        if (lane < nw) warp_sums[lane] = s;
    }
    __syncthreads();
    const int base = w ? warp_sums[w - 1] : 0;
    if (total) *total = warp_sums[nw - 1];
    return base + inc - v;
}

}  // namespace tc

#define TC_CUDA_TRY(expr)                                                            \
    do {                                                                             \
        cudaError_t err__ = (expr);                                                  \
        if (err__ != cudaSuccess) {                                                  \
            ::tc::set_error(::TC_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__,       \
                            #expr, cudaGetErrorString(err__));                       \
            return ::TC_ERR_CUDA;                                                    \
        }                                                                            \
    } while (0)

// Every kernel launch site is followed by TC_KERNEL_CHECK(), which also counts the launch.
#define TC_KERNEL_CHECK()          \
    do {                           \
        ++::tc::g_launches;        \
        TC_CUDA_TRY(cudaGetLastError()); \
    } while (0)

namespace tc {
// Kernel launches issued by this thread since the counter was last reset (per solve).
extern thread_local long long g_launches;
// Records status and message for treecode_last_status / treecode_last_error (thread-local).
void set_error(int status, const char *fmt, ...);
}
