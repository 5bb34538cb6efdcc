// sort.cu -- bounding square, Morton keys, LSD radix sort with a stable permutation, and the
// source gather.  Restates drivers/sort-sources.cpp:23-132 of the reference.
//
// Data flow per solve (N sources, all FP64 SoA in HBM):
//   k_bbox          x, y           -> Frame (xmin, ymin, ext, scale)       2 x 8 B/src read
//   k_keys          x, y, Frame    -> keys (30-bit Morton)                 16 B read, 4 B write
//   radix sort      keys (+ index) -> sorted keys, permutation             4 onesweep passes
//   k_gather        x, y, v, perm  -> sorted x, y, v                       24 B gathered, 24 B written
//
// The radix sort is a one-pass-per-digit ("onesweep") LSD sort: every CTA ranks a tile of
// 4096 keys in shared memory with warp-level match_any, publishes its per-digit counts, and
// finds its global offsets by a decoupled look-back over the tiles before it.  Tiles take
// their ids from an atomic counter, so each waits only on tiles that already run; the waits
// are bounded and raise DEVERR_SPIN_LIMIT instead of hanging.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <mutex>

#include "tc_internal.h"

namespace tc {

// ---------------------------------------------------------------------------- bbox
constexpr int BBOX_THREADS = 256;

__device__ __forceinline__ void warp_minmax(double &a, double &b, double &c, double &d) {
    for (int m = 16; m; m >>= 1) {
        a = fmin(a, shfl_xor_d(a, m));
        b = fmax(b, shfl_xor_d(b, m));
        c = fmin(c, shfl_xor_d(c, m));
        d = fmax(d, shfl_xor_d(d, m));
    }
}

// Per-CTA min/max, then the last CTA to finish reduces the partials and derives the frame.
// Initial extrema follow upward-common.ispc:132 (min 1e13, max 0) and sort-sources.cpp:48.
__global__ __launch_bounds__(BBOX_THREADS) void k_bbox(const double *__restrict__ x,
                                                       const double *__restrict__ y, int n,
                                                       double4 *partials, unsigned *done,
                                                       Frame *frame) {
    double xmi = 1e13, xma = 0, ymi = 1e13, yma = 0;
    auto take = [&](double xv, double yv) {
        xmi = fmin(xmi, xv);
        xma = fmax(xma, xv);
        ymi = fmin(ymi, yv);
        yma = fmax(yma, yv);
    };
    const int gid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0) {
        // 16-byte loads, two pairs per thread in flight
        const double2 *x2 = reinterpret_cast<const double2 *>(x);
        const double2 *y2 = reinterpret_cast<const double2 *>(y);
        const int n2 = n / 2;
        int i = gid;
        for (; i + stride < n2; i += 2 * stride) {
            const double2 a = x2[i], b = y2[i], c = x2[i + stride], e = y2[i + stride];
            take(a.x, b.x);
            take(a.y, b.y);
            take(c.x, e.x);
            take(c.y, e.y);
        }
        if (i < n2) {
            const double2 a = x2[i], b = y2[i];
            take(a.x, b.x);
            take(a.y, b.y);
        }
        if ((n & 1) && gid == 0) take(x[n - 1], y[n - 1]);
    } else {
        for (int i = gid; i < n; i += stride) take(x[i], y[i]);
    }
    warp_minmax(xmi, xma, ymi, yma);
    __shared__ double4 s[BBOX_THREADS / 32];
    __shared__ bool last;
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) s[w] = make_double4(xmi, xma, ymi, yma);
    __syncthreads();
    if (threadIdx.x == 0) {
        double4 r = s[0];
        for (int i = 1; i < BBOX_THREADS / 32; ++i) {
            r.x = fmin(r.x, s[i].x); r.y = fmax(r.y, s[i].y);
            r.z = fmin(r.z, s[i].z); r.w = fmax(r.w, s[i].w);
        }
        partials[blockIdx.x] = r;
        __threadfence();
        last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    xmi = 1e13; xma = 0; ymi = 1e13; yma = 0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
        const double2 ra = __ldcg(reinterpret_cast<const double2 *>(&partials[i]));
        const double2 rb = __ldcg(reinterpret_cast<const double2 *>(&partials[i]) + 1);
        xmi = fmin(xmi, ra.x); xma = fmax(xma, ra.y);
        ymi = fmin(ymi, rb.x); yma = fmax(yma, rb.y);
    }
    warp_minmax(xmi, xma, ymi, yma);
    __syncthreads();
    if (lane_id() == 0) s[w] = make_double4(xmi, xma, ymi, yma);
    __syncthreads();
    if (threadIdx.x == 0) {
        double4 r = s[0];
        for (int i = 1; i < BBOX_THREADS / 32; ++i) {
            r.x = fmin(r.x, s[i].x); r.y = fmax(r.y, s[i].y);
            r.z = fmin(r.z, s[i].z); r.w = fmax(r.w, s[i].w);
        }
        // sort-sources.cpp:98-110, with the arithmetic the compiled reference executes:
        // ext = max(ex, ey) * (1 + 2 eps); xmin -= eps * ext; keys use (1/ext) * 2^15.
        const double eps = 10000.0 * DBL_EPSILON;
        const double ext0 = __dsub_rn(r.y, r.x);
        const double ext1 = __dsub_rn(r.w, r.z);
        const double ext = __dmul_rn(ext0 < ext1 ? ext1 : ext0, 1.0 + 2.0 * eps);
        Frame f;
        f.xmin = __dsub_rn(r.x, __dmul_rn(eps, ext));
        f.ymin = __dsub_rn(r.z, __dmul_rn(eps, ext));
        f.ext = ext;
        f.scale = __dmul_rn(__ddiv_rn(1.0, ext), (double)(1 << LMAX));
        *frame = f;
        *done = 0;
    }
}

// ---------------------------------------------------------------------------- keys
// sort-sources.cpp:114-137: x = floor((x - xmin) * scale), bits interleaved, x on even bits.
__device__ __forceinline__ int quantize(double v, double vmin, double scale) {
    return (int)floor(__dmul_rn(__dsub_rn(v, vmin), scale));
}

__global__ void k_keys(const double *__restrict__ x, const double *__restrict__ y, int n,
                       const Frame *__restrict__ frame, int *__restrict__ keys) {
    const Frame f = *frame;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int kx = quantize(x[i], f.xmin, f.scale);
        const int ky = quantize(y[i], f.ymin, f.scale);
        keys[i] = spread_bits(kx) | (spread_bits(ky) << 1);
    }
}

// Target keys in the source frame, clamped to the quantisation range (targets may lie outside
// the sources' square).  Used only to group nearby targets; it does not affect results.
__global__ void k_target_keys(const double *__restrict__ x, const double *__restrict__ y, int n,
                              const Frame *__restrict__ frame, int *__restrict__ keys) {
    const Frame f = *frame;
    const double hi = (double)((1 << LMAX) - 1);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double qx = floor((x[i] - f.xmin) * f.scale);
        double qy = floor((y[i] - f.ymin) * f.scale);
        qx = fmin(fmax(qx, 0.0), hi);
        qy = fmin(fmax(qy, 0.0), hi);
        if (qx != qx) qx = 0;
        if (qy != qy) qy = 0;
        keys[i] = spread_bits((int)qx) | (spread_bits((int)qy) << 1);
    }
}

__global__ void k_gather3(const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ v, const int *__restrict__ perm, int n,
                          double *__restrict__ xs, double *__restrict__ ys,
                          double *__restrict__ vs, unsigned *err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int j = perm[i];
        if ((unsigned)j >= (unsigned)n) {
            atomicOr(err, DEVERR_BOUNDS);
            continue;
        }
        xs[i] = x[j];
        ys[i] = y[j];
        vs[i] = v[j];
    }
}

// ---------------------------------------------------------------------------- radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_RADIX = 256;
constexpr unsigned RS_FLAG_AGG = 1u << 30;
constexpr unsigned RS_FLAG_INC = 2u << 30;
constexpr unsigned RS_VALMASK = (1u << 30) - 1;
constexpr int RS_SPIN_LIMIT = 1 << 22;
constexpr int RS_MAX_PASSES = 4;

// Histograms of every 8-bit digit of the keys, in one read.
__global__ __launch_bounds__(256) void k_hist(const int *__restrict__ keys, int n, int npasses,
                                              int *__restrict__ hist) {
    __shared__ int s[RS_MAX_PASSES][RS_RADIX];
    for (int i = threadIdx.x; i < RS_MAX_PASSES * RS_RADIX; i += blockDim.x) (&s[0][0])[i] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned k = (unsigned)keys[i];
        for (int p = 0; p < npasses; ++p) atomicAdd(&s[p][(k >> (8 * p)) & 0xFF], 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npasses * RS_RADIX; i += blockDim.x) {
        const int c = (&s[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// Morton keys of the sources and the histograms of every 8-bit digit of them, in one pass
// (k_keys followed by k_hist, without reading the keys back).
__global__ __launch_bounds__(256) void k_keys_hist(const double *__restrict__ x,
                                                   const double *__restrict__ y, int n,
                                                   const Frame *__restrict__ frame,
                                                   int *__restrict__ keys, int npasses,
                                                   int *__restrict__ hist) {
    __shared__ int s[RS_MAX_PASSES][RS_RADIX];
    for (int i = threadIdx.x; i < RS_MAX_PASSES * RS_RADIX; i += blockDim.x) (&s[0][0])[i] = 0;
    __syncthreads();
    const Frame f = *frame;
    auto key_of = [&](double xv, double yv) {
        const int k = spread_bits(quantize(xv, f.xmin, f.scale)) |
                      (spread_bits(quantize(yv, f.ymin, f.scale)) << 1);
        for (int p = 0; p < npasses; ++p) atomicAdd(&s[p][((unsigned)k >> (8 * p)) & 0xFF], 1);
        return k;
    };
    const int gid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0 &&
        (reinterpret_cast<uintptr_t>(keys) & 7) == 0) {
        // 16-byte loads and 8-byte stores: two sources per thread and step
        const double2 *x2 = reinterpret_cast<const double2 *>(x);
        const double2 *y2 = reinterpret_cast<const double2 *>(y);
        int2 *k2 = reinterpret_cast<int2 *>(keys);
        for (int i = gid; i < n / 2; i += stride) {
            const double2 a = x2[i], b = y2[i];
            k2[i] = make_int2(key_of(a.x, b.x), key_of(a.y, b.y));
        }
        if ((n & 1) && gid == 0) keys[n - 1] = key_of(x[n - 1], y[n - 1]);
    } else {
        for (int i = gid; i < n; i += stride) keys[i] = key_of(x[i], y[i]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npasses * RS_RADIX; i += blockDim.x) {
        const int c = (&s[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

__global__ __launch_bounds__(RS_RADIX) void k_hist_scan(const int *__restrict__ hist,
                                                        int *__restrict__ offsets) {
    const int p = blockIdx.x;
    const int v = hist[p * RS_RADIX + threadIdx.x];
    offsets[p * RS_RADIX + threadIdx.x] = block_exclusive_scan(v, nullptr);
}

__device__ __forceinline__ unsigned ld_volatile(const unsigned *p) {
    return *(const volatile unsigned *)p;
}

// Exclusive prefix of digit d over the tiles before `tile` (decoupled look-back): walk back
// over the predecessors' statuses, adding aggregates, until the first inclusive prefix.  A
// predecessor that has published nothing yet is read again; the number of such reads is
// bounded (DEVERR_SPIN_LIMIT).  (Reading several predecessors per step measured slower.)
__device__ __forceinline__ int lookback(const unsigned *status, int tile, int d, unsigned *err) {
    int excl = 0;
    int spins = 0;
    for (int j = tile - 1; j >= 0;) {
        const unsigned s = ld_volatile(status + (size_t)j * RS_RADIX + d);
        const unsigned flag = s & ~RS_VALMASK;
        if (flag == 0) {
            if (++spins > RS_SPIN_LIMIT) {
                atomicOr(err, DEVERR_SPIN_LIMIT);
                break;
            }
            continue;
        }
        excl += (int)(s & RS_VALMASK);
        if (flag == RS_FLAG_INC) break;
        --j;
    }
    return excl;
}

__global__ __launch_bounds__(RS_THREADS) void k_onesweep(
    const int *__restrict__ keys_in, const int *__restrict__ vals_in, int *__restrict__ keys_out,
    int *__restrict__ vals_out, int n, int shift, const int *__restrict__ digit_offsets,
    unsigned *status, int *tile_counter, unsigned *err) {
    __shared__ int s_keys[RS_TILE];
    __shared__ int s_vals[RS_TILE];
    __shared__ int s_whist[RS_WARPS][RS_RADIX];
    __shared__ int s_tile_start[RS_RADIX];
    __shared__ int s_global[RS_RADIX];
    __shared__ int s_tile;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1);
    for (int i = tid; i < RS_WARPS * RS_RADIX; i += RS_THREADS) (&s_whist[0][0])[i] = 0;
    __syncthreads();
    const int tile = s_tile;
    const int tile_base = tile * RS_TILE;
    const int warp_base = tile_base + warp * (RS_ITEMS * 32);

    int key[RS_ITEMS], val[RS_ITEMS], rank[RS_ITEMS];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const int idx = warp_base + k * 32 + lane;
        const bool valid = idx < n;
        key[k] = valid ? keys_in[idx] : 0;
        val[k] = valid ? (vals_in ? vals_in[idx] : idx) : 0;
    }

    // Stable rank within the warp: items are visited in their original order (k, lane).
    const unsigned lt = lanemask_lt();
    int *hist = s_whist[warp];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const int idx = warp_base + k * 32 + lane;
        const bool valid = idx < n;
        const unsigned vmask = __ballot_sync(FULL_MASK, valid);
        const int d = (key[k] >> shift) & 0xFF;
        unsigned peers = 0;
        if (valid) peers = __match_any_sync(vmask, d);
        const int old = valid ? hist[d] : 0;
        __syncwarp();
        if (valid && (peers & lt) == 0) hist[d] = old + __popc(peers);
        __syncwarp();
        rank[k] = old + __popc(peers & lt);
    }
    __syncthreads();

    // Thread `tid` owns digit `tid`: exclusive prefix over warps and the tile's count.
    const int d = tid;
    int total = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) {
        const int c = s_whist[w][d];
        s_whist[w][d] = total;
        total += c;
    }

    // Decoupled look-back for this digit.
    unsigned *mine = status + (size_t)tile * RS_RADIX + d;
    int excl = 0;
    if (tile == 0) {
        atomicExch(mine, RS_FLAG_INC | (unsigned)total);
    } else {
        atomicExch(mine, RS_FLAG_AGG | (unsigned)total);
        excl = lookback(status, tile, d, err);
        atomicExch(mine, RS_FLAG_INC | (unsigned)(excl + total));
    }

    const int start = block_exclusive_scan(total, nullptr);
    s_tile_start[d] = start;
    s_global[d] = digit_offsets[d] + excl - start;
    __syncthreads();

#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const int idx = warp_base + k * 32 + lane;
        if (idx < n) {
            const int dk = (key[k] >> shift) & 0xFF;
            const int pos = s_tile_start[dk] + s_whist[warp][dk] + rank[k];
            if ((unsigned)pos >= (unsigned)RS_TILE) {
                atomicOr(err, DEVERR_BOUNDS);
                continue;
            }
            s_keys[pos] = key[k];
            s_vals[pos] = val[k];
        }
    }
    __syncthreads();

    const int tile_n = min(RS_TILE, n - tile_base);
    for (int j = tid; j < tile_n; j += RS_THREADS) {
        const int kk = s_keys[j];
        const int g = s_global[(kk >> shift) & 0xFF] + j;
        if ((unsigned)g >= (unsigned)n) {
            atomicOr(err, DEVERR_BOUNDS);
            continue;
        }
        keys_out[g] = kk;
        vals_out[g] = s_vals[j];
    }
}

// L2 prefetch of [p, p + bytes) rounded inwards to 16-byte bounds (a hint: no data moves to
// the SM, nothing is written).
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
    const uintptr_t a = (reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + bytes) & ~uintptr_t(15);
    if (e > a)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(a), "r"((unsigned)(e - a))
                     : "memory");
}

// The same pass for the sources, carrying the input index, coordinates and values along with
// the key, so that the sorted x/y/v come out of the last pass without a random gather over the
// whole array (~300 B of DRAM traffic per source on HBM, against 28 + 28 B here).
//   * tiles of 2048 sources, 256 threads, 8 items per thread; three CTAs fit one SM;
//   * at the start of a tile one thread asks for the tile's index/x/y/v ranges to be brought
//     into L2 (cp.async.bulk.prefetch), so their DRAM latency overlaps ranking and look-back;
//   * once the local positions are known every item's index, x, y and v are loaded together
//     (32 loads in flight per thread, served by L2) and placed in sorted order in shared memory;
//   * one output loop writes all five arrays, slot j going to s_global[digit] + j.
constexpr int XYV_THREADS = 256;
constexpr int XYV_WARPS = XYV_THREADS / 32;
constexpr int XYV_ITEMS = 8;
constexpr int XYV_TILE = XYV_THREADS * XYV_ITEMS;
constexpr size_t XYV_SMEM = (size_t)XYV_TILE * (2 * sizeof(int) + 3 * sizeof(double)) +
                            (size_t)XYV_WARPS * RS_RADIX * sizeof(int) + 2 * RS_RADIX * sizeof(int) +
                            16;

__global__ __launch_bounds__(XYV_THREADS) void k_onesweep_xyv(
    const int *__restrict__ keys_in, const int *__restrict__ idx_in,
    const double *__restrict__ x_in, const double *__restrict__ y_in,
    const double *__restrict__ v_in, int *__restrict__ keys_out, int *__restrict__ idx_out,
    double *__restrict__ x_out, double *__restrict__ y_out, double *__restrict__ v_out, int n,
    int shift, const int *__restrict__ digit_offsets, unsigned *status, int *tile_counter,
    unsigned *err) {
    extern __shared__ __align__(16) unsigned char xyv_smem[];
    double *s_x = reinterpret_cast<double *>(xyv_smem);
    double *s_y = s_x + XYV_TILE;
    double *s_v = s_y + XYV_TILE;
    int *s_keys = reinterpret_cast<int *>(s_v + XYV_TILE);
    int *s_idx = s_keys + XYV_TILE;
    int(*s_whist)[RS_RADIX] = reinterpret_cast<int(*)[RS_RADIX]>(s_idx + XYV_TILE);
    int *s_tile_start = &s_whist[XYV_WARPS][0];
    int *s_global = s_tile_start + RS_RADIX;
    int *s_tile = s_global + RS_RADIX;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) *s_tile = atomicAdd(tile_counter, 1);
    for (int i = tid; i < XYV_WARPS * RS_RADIX; i += XYV_THREADS) (&s_whist[0][0])[i] = 0;
    __syncthreads();
    const int tile = *s_tile;
    const int tile_base = tile * XYV_TILE;
    const int tile_n = min(XYV_TILE, n - tile_base);
    const int warp_base = tile_base + warp * (XYV_ITEMS * 32);
    if (tid == 0) {
        prefetch_l2(x_in + tile_base, sizeof(double) * tile_n);
        prefetch_l2(y_in + tile_base, sizeof(double) * tile_n);
        prefetch_l2(v_in + tile_base, sizeof(double) * tile_n);
        if (idx_in) prefetch_l2(idx_in + tile_base, sizeof(int) * tile_n);
    }

    int key[XYV_ITEMS], pos[XYV_ITEMS];
#pragma unroll
    for (int k = 0; k < XYV_ITEMS; ++k) {
        const int idx = warp_base + k * 32 + lane;
        key[k] = idx < n ? keys_in[idx] : 0;
    }

    // stable rank within the warp, items visited in their original order (k, lane)
    const unsigned lt = lanemask_lt();
    int *hist = s_whist[warp];
#pragma unroll
    for (int k = 0; k < XYV_ITEMS; ++k) {
        const int idx = warp_base + k * 32 + lane;
        const bool valid = idx < n;
        const unsigned vmask = __ballot_sync(FULL_MASK, valid);
        const int d = (key[k] >> shift) & 0xFF;
        unsigned peers = 0;
        if (valid) peers = __match_any_sync(vmask, d);
        const int old = valid ? hist[d] : 0;
        __syncwarp();
        if (valid && (peers & lt) == 0) hist[d] = old + __popc(peers);
        __syncwarp();
        pos[k] = old + __popc(peers & lt);
    }
    __syncthreads();

    const int d = tid;   // one digit per thread
    int total = 0;
#pragma unroll
    for (int w = 0; w < XYV_WARPS; ++w) {
        const int c = s_whist[w][d];
        s_whist[w][d] = total;
        total += c;
    }
    unsigned *mine = status + (size_t)tile * RS_RADIX + d;
    int excl = 0;
    if (tile == 0) {
        atomicExch(mine, RS_FLAG_INC | (unsigned)total);
    } else {
        atomicExch(mine, RS_FLAG_AGG | (unsigned)total);
        excl = lookback(status, tile, d, err);
        atomicExch(mine, RS_FLAG_INC | (unsigned)(excl + total));
    }
    const int start = block_exclusive_scan(total, nullptr);
    s_tile_start[d] = start;
    s_global[d] = digit_offsets[d] + excl - start;
    __syncthreads();

    // every item to its sorted slot in shared memory, with its index, x, y and v
#pragma unroll
    for (int k = 0; k < XYV_ITEMS; ++k) {
        const int idx = warp_base + k * 32 + lane;
        if (idx < n) {
            const int dk = (key[k] >> shift) & 0xFF;
            const int p = s_tile_start[dk] + s_whist[warp][dk] + pos[k];
            if ((unsigned)p >= (unsigned)tile_n) {
                atomicOr(err, DEVERR_BOUNDS);
            } else {
                s_keys[p] = key[k];
                s_idx[p] = idx_in ? __ldg(idx_in + idx) : idx;
                s_x[p] = __ldg(x_in + idx);
                s_y[p] = __ldg(y_in + idx);
                s_v[p] = __ldg(v_in + idx);
            }
        }
    }
    __syncthreads();

    // slot j goes to s_global[digit] + j: runs of equal digits are consecutive in memory
#pragma unroll 4
    for (int j = tid; j < tile_n; j += XYV_THREADS) {
        const int kj = s_keys[j];
        const int g = s_global[(kj >> shift) & 0xFF] + j;
        if ((unsigned)g >= (unsigned)n) {
            atomicOr(err, DEVERR_BOUNDS);
            continue;
        }
        keys_out[g] = kj;
        idx_out[g] = s_idx[j];
        x_out[g] = s_x[j];
        y_out[g] = s_y[j];
        v_out[g] = s_v[j];
    }
}

static int grid_for(int n, int threads, int per_sm = 8) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long g = ((long long)n + threads - 1) / threads;
    long long cap = (long long)sms * per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

int radix_sort_pairs(Context &c, const int *keys_in, const int *vals_in, int n, int nbits,
                     int *keys_a, int *vals_a, int *keys_b, int *vals_b, int **keys_out,
                     int **vals_out) {
    if (n >= (1 << 30)) {
        set_error(TC_ERR_INVALID, "radix sort supports fewer than 2^30 keys (got %d)", n);
        return TC_ERR_INVALID;
    }
    const int npasses = (nbits + 7) / 8;
    const int ntiles = (n + RS_TILE - 1) / RS_TILE;
    int *hist, *counter;
    unsigned *status;
    int rc;
    if ((rc = ensure(c, S_RS_HIST, 2 * RS_MAX_PASSES * RS_RADIX, &hist))) return rc;
    if ((rc = ensure(c, S_RS_COUNTER, RS_MAX_PASSES, &counter))) return rc;
    if ((rc = ensure(c, S_RS_STATUS, (size_t)RS_MAX_PASSES * ntiles * RS_RADIX, &status))) return rc;
    int *offsets = hist + RS_MAX_PASSES * RS_RADIX;
    TC_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(int) * RS_MAX_PASSES * RS_RADIX, c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int) * RS_MAX_PASSES, c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned) * (size_t)npasses * ntiles * RS_RADIX,
                                c.stream));
    k_hist<<<grid_for(n, 256, 4), 256, 0, c.stream>>>(keys_in, n, npasses, hist);
    TC_KERNEL_CHECK();
    k_hist_scan<<<npasses, RS_RADIX, 0, c.stream>>>(hist, offsets);
    TC_KERNEL_CHECK();
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);

    const int *ki = keys_in, *vi = vals_in;
    int *ko = keys_a, *vo = vals_a;
    for (int p = 0; p < npasses; ++p) {
        k_onesweep<<<ntiles, RS_THREADS, 0, c.stream>>>(ki, vi, ko, vo, n, 8 * p,
                                                         offsets + p * RS_RADIX,
                                                         status + (size_t)p * ntiles * RS_RADIX,
                                                         counter + p, err);
        TC_KERNEL_CHECK();
        ki = ko;
        vi = vo;
        if (ko == keys_a) { ko = keys_b; vo = vals_b; }
        else { ko = keys_a; vo = vals_a; }
    }
    *keys_out = const_cast<int *>(ki);
    *vals_out = const_cast<int *>(vi);
    return TC_OK;
}

// ---------------------------------------------------------------------------- scan
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__global__ __launch_bounds__(SCAN_THREADS) void k_scan_reduce(const int *__restrict__ in, int n,
                                                             int *__restrict__ block_sums) {
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i)
        if (base + i < n) s += in[base + i];
    int total;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ __launch_bounds__(SCAN_THREADS) void k_scan_blocks(int *block_sums, int nb,
                                                             int *out_total) {
    // one CTA: each thread scans a contiguous chunk of the block sums
    const int per = (nb + SCAN_THREADS - 1) / SCAN_THREADS;
    const int b0 = threadIdx.x * per;
    int s = 0;
    for (int i = 0; i < per; ++i)
        if (b0 + i < nb) s += block_sums[b0 + i];
    int total;
    int run = block_exclusive_scan(s, &total);
    for (int i = 0; i < per; ++i)
        if (b0 + i < nb) {
            const int v = block_sums[b0 + i];
            block_sums[b0 + i] = run;
            run += v;
        }
    if (threadIdx.x == 0) *out_total = total;
}

__global__ __launch_bounds__(SCAN_THREADS) void k_scan_apply(const int *__restrict__ in, int n,
                                                            const int *__restrict__ block_offs,
                                                            int *__restrict__ out) {
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        v[i] = base + i < n ? in[base + i] : 0;
        s += v[i];
    }
    int run = block_exclusive_scan(s, nullptr) + block_offs[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i)
        if (base + i < n) {
            out[base + i] = run;
            run += v[i];
        }
}

int exclusive_scan(Context &c, const int *d_in, int *d_out, int n) {
    const int nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    int *bs;
    int rc;
    if ((rc = ensure(c, S_SCAN_BLOCKS, (size_t)nb + 1, &bs))) return rc;
    if (n == 0) {
        TC_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(int), c.stream));
        return TC_OK;
    }
    k_scan_reduce<<<nb, SCAN_THREADS, 0, c.stream>>>(d_in, n, bs);
    TC_KERNEL_CHECK();
    k_scan_blocks<<<1, SCAN_THREADS, 0, c.stream>>>(bs, nb, d_out + n);
    TC_KERNEL_CHECK();
    k_scan_apply<<<nb, SCAN_THREADS, 0, c.stream>>>(d_in, n, bs, d_out);
    TC_KERNEL_CHECK();
    return TC_OK;
}

// ---------------------------------------------------------------------------- drivers
int sort_sources(Context &c, const double *x, const double *y, const double *v, int n) {
    int rc;
    double *xs, *ys, *vs;
    int *keys, *perm, *keys2, *perm2;
    Frame *frame;
    double4 *partials;
    if ((rc = ensure(c, S_XS, n, &xs)) || (rc = ensure(c, S_YS, n, &ys)) ||
        (rc = ensure(c, S_VS, n, &vs)) || (rc = ensure(c, S_KEYS, n, &keys)) ||
        (rc = ensure(c, S_PERM, n, &perm)) || (rc = ensure(c, S_KEYS2, n, &keys2)) ||
        (rc = ensure(c, S_PERM2, n, &perm2)))
        return rc;
    // frame + bbox partials + completion counter share one small buffer
    const int gb = grid_for(n, BBOX_THREADS, 8);
    if ((rc = ensure(c, S_FRAME, sizeof(Frame) + sizeof(double4) * (gb + 1) + 64, (char **)&frame)))
        return rc;
    partials = reinterpret_cast<double4 *>(reinterpret_cast<char *>(frame) + 64);
    unsigned *done = reinterpret_cast<unsigned *>(partials + gb);
    TC_CUDA_TRY(cudaMemsetAsync(done, 0, sizeof(unsigned), c.stream));
    k_bbox<<<gb, BBOX_THREADS, 0, c.stream>>>(x, y, n, partials, done, frame);
    TC_KERNEL_CHECK();

    // four 8-bit passes carrying (index, x, y, v); the ping-pong
    // input -> tmp -> sorted -> tmp -> sorted ends in keys/perm/xs/ys/vs
    if (n >= (1 << 30)) {
        set_error(TC_ERR_INVALID, "too many sources for the radix sort (%d)", n);
        return TC_ERR_INVALID;
    }
    double *x2, *y2, *v2;
    int *hist, *counter;
    unsigned *status;
    const int npasses = (2 * LMAX + 7) / 8;
    const int ntiles = (n + XYV_TILE - 1) / XYV_TILE;
    if ((rc = ensure(c, S_X2, n, &x2)) || (rc = ensure(c, S_Y2, n, &y2)) ||
        (rc = ensure(c, S_V2, n, &v2)) ||
        (rc = ensure(c, S_RS_HIST, 2 * RS_MAX_PASSES * RS_RADIX, &hist)) ||
        (rc = ensure(c, S_RS_COUNTER, RS_MAX_PASSES, &counter)) ||
        (rc = ensure(c, S_RS_STATUS, (size_t)RS_MAX_PASSES * ntiles * RS_RADIX, &status)))
        return rc;
    int *offsets = hist + RS_MAX_PASSES * RS_RADIX;
    TC_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(int) * RS_MAX_PASSES * RS_RADIX, c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int) * RS_MAX_PASSES, c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned) * (size_t)npasses * ntiles * RS_RADIX,
                                c.stream));
    k_keys_hist<<<grid_for(n, 256, 8), 256, 0, c.stream>>>(x, y, n, frame, keys, npasses, hist);
    TC_KERNEL_CHECK();
    k_hist_scan<<<npasses, RS_RADIX, 0, c.stream>>>(hist, offsets);
    TC_KERNEL_CHECK();
    static const cudaError_t attr_rc = cudaFuncSetAttribute(
        k_onesweep_xyv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XYV_SMEM);
    TC_CUDA_TRY(attr_rc);
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);
    static_assert((2 * LMAX + 7) / 8 % 2 == 0, "an even number of passes ends in the sorted arrays");
    for (int p = 0; p < npasses; ++p) {
        const bool odd = p & 1;
        const int *ki = odd ? keys2 : keys;
        const int *ii = p == 0 ? nullptr : (odd ? perm2 : perm);
        const double *xi = p == 0 ? x : (odd ? x2 : xs);
        const double *yi = p == 0 ? y : (odd ? y2 : ys);
        const double *vi = p == 0 ? v : (odd ? v2 : vs);
        int *ko = odd ? keys : keys2, *io = odd ? perm : perm2;
        double *xo = odd ? xs : x2, *yo = odd ? ys : y2, *vo = odd ? vs : v2;
        k_onesweep_xyv<<<ntiles, XYV_THREADS, XYV_SMEM, c.stream>>>(
            ki, ii, xi, yi, vi, ko, io, xo, yo, vo, n, 8 * p, offsets + p * RS_RADIX,
            status + (size_t)p * ntiles * RS_RADIX, counter + p, err);
        TC_KERNEL_CHECK();
    }
    c.nsrc = n;
    return TC_OK;
}

int target_keys(Context &c, const double *xt, const double *yt, int m, int *keys, int *idx) {
    (void)idx;
    Frame *frame = slot_ptr<Frame>(c, S_FRAME);
    k_target_keys<<<grid_for(m, 256), 256, 0, c.stream>>>(xt, yt, m, frame, keys);
    TC_KERNEL_CHECK();
    return TC_OK;
}

// ---------------------------------------------------------------------------- allocation-free
// Source sort for callers that cannot allocate device memory.  Everything the sort needs
// besides the caller's inputs and outputs -- the second key/permutation buffer of the
// ping-pong passes, the per-tile look-back words, the digit histograms, the tile counters,
// the bounding-box partials and the error word -- lives in one static device array of fixed
// size, so a call makes no cudaMalloc/cudaFree and no other allocating call.
constexpr int NOALLOC_MAX_SOURCES = 1 << 20;
constexpr int NA_MAX_TILES = (NOALLOC_MAX_SOURCES + RS_TILE - 1) / RS_TILE;
constexpr int NA_MAX_BBOX_BLOCKS = 4096;
constexpr size_t NA_OFF_KEYS = 0;
constexpr size_t NA_OFF_PERM = NA_OFF_KEYS + sizeof(int) * NOALLOC_MAX_SOURCES;
constexpr size_t NA_OFF_STATUS = NA_OFF_PERM + sizeof(int) * NOALLOC_MAX_SOURCES;
constexpr size_t NA_OFF_HIST =
    NA_OFF_STATUS + sizeof(unsigned) * RS_MAX_PASSES * NA_MAX_TILES * RS_RADIX;
constexpr size_t NA_OFF_CTR = NA_OFF_HIST + sizeof(int) * 2 * RS_MAX_PASSES * RS_RADIX;
constexpr size_t NA_OFF_ERR = NA_OFF_CTR + 256;
constexpr size_t NA_OFF_DONE = NA_OFF_ERR + 256;
constexpr size_t NA_OFF_PARTIALS = NA_OFF_DONE + 256;
constexpr size_t NA_BYTES = NA_OFF_PARTIALS + sizeof(double4) * NA_MAX_BBOX_BLOCKS;  // ~9.2 MB

// One copy per device that loads the library, held until the process exits.  In host code
// the name is only a host-side handle: kernels get the device address from
// cudaGetSymbolAddress (noalloc_scratch_base), never the symbol itself.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

static unsigned char *noalloc_scratch_base(int device) {
    constexpr int MAX_DEVICES = 64;
    static std::mutex mu;
    static void *addr[MAX_DEVICES] = {};
    if (device < 0 || device >= MAX_DEVICES) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            set_error(TC_ERR_CUDA, "tc_sort_sources_noalloc: cudaGetSymbolAddress failed: %s",
                      cudaGetErrorString(e));
            return nullptr;
        }
        addr[device] = p;
    }
    return static_cast<unsigned char *>(addr[device]);
}

}  // namespace tc

extern "C" TC_API int tc_sort_sources_noalloc(const double *xsources, const double *ysources,
                                              const double *sourcevalues, int nsources,
                                              int *keys, int *perm, double *xsorted,
                                              double *ysorted, double *vsorted, double *frame,
                                              void *cuda_stream) {
    using namespace tc;
    set_error(TC_OK, "");
    const int n = nsources;
    if (n < 0 || n > NOALLOC_MAX_SOURCES) {
        set_error(TC_ERR_INVALID,
                  "tc_sort_sources_noalloc: nsources = %d is outside [0, %d], the size of its "
                  "fixed scratch array", n, NOALLOC_MAX_SOURCES);
        return TC_ERR_INVALID;
    }
    if (n == 0) return TC_OK;
    if (!xsources || !ysources || !sourcevalues || !keys || !perm || !xsorted || !ysorted ||
        !vsorted || !frame) {
        set_error(TC_ERR_INVALID, "tc_sort_sources_noalloc: NULL array argument");
        return TC_ERR_INVALID;
    }
    int dev = 0;
    TC_CUDA_TRY(cudaGetDevice(&dev));
    unsigned char *base = noalloc_scratch_base(dev);
    if (!base) {
        if (treecode_last_status() == TC_OK)
            set_error(TC_ERR_INVALID, "tc_sort_sources_noalloc: device %d not supported", dev);
        return treecode_last_status();
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    int *keys_tmp = reinterpret_cast<int *>(base + NA_OFF_KEYS);
    int *perm_tmp = reinterpret_cast<int *>(base + NA_OFF_PERM);
    unsigned *status = reinterpret_cast<unsigned *>(base + NA_OFF_STATUS);
    int *hist = reinterpret_cast<int *>(base + NA_OFF_HIST);
    int *offsets = hist + RS_MAX_PASSES * RS_RADIX;
    int *counter = reinterpret_cast<int *>(base + NA_OFF_CTR);
    unsigned *err = reinterpret_cast<unsigned *>(base + NA_OFF_ERR);
    unsigned *done = reinterpret_cast<unsigned *>(base + NA_OFF_DONE);
    double4 *partials = reinterpret_cast<double4 *>(base + NA_OFF_PARTIALS);
    Frame *fr = reinterpret_cast<Frame *>(frame);

    // The array keeps the previous call's contents: clear what has to start at zero.
    const int npasses = (2 * LMAX + 7) / 8;
    const int ntiles = (n + RS_TILE - 1) / RS_TILE;
    TC_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(unsigned), s));
    TC_CUDA_TRY(cudaMemsetAsync(done, 0, sizeof(unsigned), s));
    TC_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(int) * RS_MAX_PASSES * RS_RADIX, s));
    TC_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int) * RS_MAX_PASSES, s));
    TC_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned) * (size_t)npasses * ntiles * RS_RADIX, s));

    const int gb = std::min(grid_for(n, BBOX_THREADS, 8), NA_MAX_BBOX_BLOCKS);
    k_bbox<<<gb, BBOX_THREADS, 0, s>>>(xsources, ysources, n, partials, done, fr);
    TC_KERNEL_CHECK();
    k_keys<<<grid_for(n, 256), 256, 0, s>>>(xsources, ysources, n, fr, keys);
    TC_KERNEL_CHECK();
    k_hist<<<grid_for(n, 256, 4), 256, 0, s>>>(keys, n, npasses, hist);
    TC_KERNEL_CHECK();
    k_hist_scan<<<npasses, RS_RADIX, 0, s>>>(hist, offsets);
    TC_KERNEL_CHECK();
    // keys -> tmp -> keys -> tmp -> keys: four passes end in the caller's arrays
    const int *ki = keys, *vi = nullptr;
    for (int p = 0; p < npasses; ++p) {
        int *ko = (p & 1) ? keys : keys_tmp;
        int *vo = (p & 1) ? perm : perm_tmp;
        k_onesweep<<<ntiles, RS_THREADS, 0, s>>>(ki, vi, ko, vo, n, 8 * p, offsets + p * RS_RADIX,
                                                  status + (size_t)p * ntiles * RS_RADIX,
                                                  counter + p, err);
        TC_KERNEL_CHECK();
        ki = ko;
        vi = vo;
    }
    static_assert((2 * LMAX + 7) / 8 % 2 == 0, "an even number of passes ends in keys/perm");
    k_gather3<<<grid_for(n, 256), 256, 0, s>>>(xsources, ysources, sourcevalues, perm, n,
                                                xsorted, ysorted, vsorted, err);
    TC_KERNEL_CHECK();
    unsigned h_err = 0;
    TC_CUDA_TRY(cudaMemcpyAsync(&h_err, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    TC_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_err) {
        set_error(h_err & DEVERR_SPIN_LIMIT ? TC_ERR_TIMEOUT : TC_ERR_CUDA,
                  "tc_sort_sources_noalloc: device error flags 0x%x", h_err);
        return treecode_last_status();
    }
    return TC_OK;
}
