// sort.cu -- bounding square, Morton keys, LSD radix sort with a stable permutation, and the
// sorted source arrays.  Restates drivers/sort-sources.cpp:23-132 of the reference.
//
// Data flow per solve (N sources, all FP64 SoA in HBM), with the values resident (the device
// entry points):
//   k_bbox            x, y        -> Frame (xmin, ymin, ext, scale)          16 B/src read
//   k_key_hist        x, y        -> histograms of the 4 key digits and of   16 B read
//                                    the 256 spatial buckets (top 8 key bits)
//   k_onesweep_items  x, y, v     -> 32-byte records (x, y, v, index) in     24 B read, 40 B written
//     (first pass)                   their buckets, items (key << 32 | slot)
//                                    sorted by the first digit
//   k_onesweep_items  items       -> items sorted by the next 8-bit digit    8 B read, 8 B written
//                                    (3 passes)
//   k_gather_sources  items, recs -> sorted keys, permutation, x, y, v       8 B + one record
//                                                                            read, 32 B written
// With values that arrive after x and y (the host entry points): k_keys_pack writes the items
// (key << 32 | index) and the histograms, four passes sort them, k_items_split writes keys and
// permutation, k_gather_xy the sorted x and y, and k_gather_v the sorted v once it is in.
//
// The radix sort is a one-pass-per-digit ("onesweep") LSD sort: every CTA counts the digits of
// a tile of items, finds its global digit offsets by a decoupled look-back over the tiles
// before it, ranks the tile in shared memory with warp digit ballots and writes it out in
// runs of equal digits.  Tiles take their ids from an atomic counter, so each waits only on
// tiles that already run; the waits are bounded and raise DEVERR_SPIN_LIMIT instead of
// hanging.  Ties keep input order, so the order is the reference's (key, index) order.
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
    pdl_begin();
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

// Target keys in the source frame, clamped to the quantisation range (targets may lie outside
// the sources' square).  Used only to group nearby targets; it does not affect results.
__global__ void k_target_keys(const double *__restrict__ x, const double *__restrict__ y, int n,
                              const Frame *__restrict__ frame, int *__restrict__ keys) {
    pdl_begin();
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

// ---------------------------------------------------------------------------- radix sort
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_RADIX = 256;
constexpr unsigned RS_FLAG_AGG = 1u << 30;
constexpr unsigned RS_FLAG_INC = 2u << 30;
constexpr unsigned RS_VALMASK = (1u << 30) - 1;
constexpr int RS_SPIN_LIMIT = DEFAULT_SPIN_LIMIT;
constexpr int RS_MAX_PASSES = 4;

// Histograms of every 8-bit digit of the keys, in one read.
__global__ __launch_bounds__(256) void k_hist(const int *__restrict__ keys, int n, int npasses,
                                              int *__restrict__ hist) {
    pdl_begin();
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

__global__ __launch_bounds__(RS_RADIX) void k_hist_scan(const int *__restrict__ hist,
                                                        int *__restrict__ offsets) {
    pdl_begin();
    const int p = blockIdx.x;
    const int v = hist[p * RS_RADIX + threadIdx.x];
    offsets[p * RS_RADIX + threadIdx.x] = block_exclusive_scan(v, nullptr);
}

__device__ __forceinline__ unsigned ld_volatile(const unsigned *p) {
    return *(const volatile unsigned *)p;
}

// The lanes of `vmask` whose 8-bit digit equals this lane's: one ballot per digit bit
// (eight cheap votes instead of one match.any, which has a much lower issue rate).
__device__ __forceinline__ unsigned digit_peers(unsigned vmask, int d) {
    unsigned peers = vmask;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        const bool bit = (d >> b) & 1;
        const unsigned bal = __ballot_sync(FULL_MASK, bit);
        peers &= bit ? bal : ~bal;
    }
    return peers;
}

// Exclusive prefix of digit d over the tiles before `tile` (decoupled look-back): walk back
// over the predecessors' statuses, adding aggregates, until the first inclusive prefix.  The
// statuses of LB_WINDOW predecessors are read at once (independent loads, each coalesced over
// the CTA's digit threads), which cuts the walk of ~17 dependent L2 round trips measured on
// 16M keys to ~6.  A predecessor that has published nothing yet is read again from there; the
// number of reads without progress is bounded by `spin_limit` (DEVERR_SPIN_LIMIT).
constexpr int LB_WINDOW = 4;

__device__ __forceinline__ int lookback(const unsigned *status, int tile, int d, unsigned *err,
                                        int spin_limit = RS_SPIN_LIMIT) {
    int excl = 0;
    int spins = 0;
    int j = tile - 1;
    while (j >= 0) {
        unsigned s[LB_WINDOW];
#pragma unroll
        for (int q = 0; q < LB_WINDOW; ++q)
            s[q] = j - q >= 0 ? ld_volatile(status + (size_t)(j - q) * RS_RADIX + d) : RS_FLAG_INC;
        int used = 0;
        bool stop = false;
#pragma unroll
        for (int q = 0; q < LB_WINDOW; ++q) {
            if (stop) continue;
            const unsigned flag = s[q] & ~RS_VALMASK;
            if (flag == 0) {
                stop = true;   // not published yet: read again from here
                continue;
            }
            excl += (int)(s[q] & RS_VALMASK);
            ++used;
            if (flag == RS_FLAG_INC) return excl;
        }
        j -= used;
        if (used == 0 && ++spins > spin_limit) {
            atomicOr(err, DEVERR_SPIN_LIMIT);
            break;
        }
    }
    return excl;
}

__global__ __launch_bounds__(RS_THREADS) void k_onesweep(
    const int *__restrict__ keys_in, const int *__restrict__ vals_in, int *__restrict__ keys_out,
    int *__restrict__ vals_out, int n, int shift, const int *__restrict__ digit_offsets,
    unsigned *status, int *tile_counter, unsigned *err) {
    pdl_begin();
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
        unsigned peers = digit_peers(vmask, d);
        if (!valid) peers = 0;
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

// ---------------------------------------------------------------------------- source sort
// The sources are sorted as 8-byte items key << 32 | payload by four onesweep passes (8-bit
// digits of the key half, 16 B of traffic per item and pass).  Ties keep input order, so the
// result is the (key, index) lexicographic order.
// k_keys_pack: the items (key << 32 | index) in input order and the histograms of the four
// digits (the late-values path and the allocation-free sort).
__global__ __launch_bounds__(256) void k_keys_pack(const double *__restrict__ x,
                                                   const double *__restrict__ y, int n,
                                                   const Frame *__restrict__ frame,
                                                   unsigned long long *__restrict__ items,
                                                   int npasses, int *__restrict__ hist) {
    pdl_begin();
    __shared__ int s[RS_MAX_PASSES][RS_RADIX];
    for (int i = threadIdx.x; i < RS_MAX_PASSES * RS_RADIX; i += blockDim.x) (&s[0][0])[i] = 0;
    __syncthreads();
    const Frame f = *frame;
    auto item_of = [&](double xv, double yv, int i) {
        const int k = spread_bits(quantize(xv, f.xmin, f.scale)) |
                      (spread_bits(quantize(yv, f.ymin, f.scale)) << 1);
        for (int p = 0; p < npasses; ++p) atomicAdd(&s[p][((unsigned)k >> (8 * p)) & 0xFF], 1);
        return ((unsigned long long)(unsigned)k << 32) | (unsigned)i;
    };
    const int gid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y) |
          reinterpret_cast<uintptr_t>(items)) & 15) == 0) {
        // 16-byte loads and stores: two sources per thread and step
        const double2 *x2 = reinterpret_cast<const double2 *>(x);
        const double2 *y2 = reinterpret_cast<const double2 *>(y);
        ulonglong2 *it2 = reinterpret_cast<ulonglong2 *>(items);
        for (int i = gid; i < n / 2; i += stride) {
            const double2 a = x2[i], b = y2[i];
            it2[i] = make_ulonglong2(item_of(a.x, b.x, 2 * i), item_of(a.y, b.y, 2 * i + 1));
        }
        if ((n & 1) && gid == 0) {
            const int i = n - 1;
            items[i] = item_of(x[i], y[i], i);
        }
    } else {
        for (int i = gid; i < n; i += stride) items[i] = item_of(x[i], y[i], i);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npasses * RS_RADIX; i += blockDim.x) {
        const int c = (&s[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// Resident values (the device entry points): the records are written by the first radix pass
// itself, grouped by the top 8 bits of the key (256 buckets, each a square of 1/16 of the
// frame's side), so that the final gather reads a window of the sorted order from a compact
// range of records, L2-resident, instead of from anywhere in HBM:
//   * k_key_hist reads x and y once and writes the histograms of the four radix digits and of
//     the top 8 key bits (the buckets);
//   * k_onesweep_items<true> (the first pass) reads x, y, v, forms the keys, claims each
//     source a record slot in its bucket (tile counts in shared memory, one global atomic per
//     tile and bucket) and writes the record (x, y, v, index); its items carry the record's
//     position, key << 32 | slot;
//   * three more passes over the items; the gather reads each record from its bucket.
// Slots within a bucket depend on tile timing, but they are only payload: the passes order by
// the key half alone and keep input order for equal keys, so the sorted keys, permutation and
// sources do not depend on them.
constexpr int NB_BUCKETS = 256;
constexpr int BUCKET_SHIFT = 2 * LMAX - 8;   // the top 8 of the 30 key bits

__device__ __forceinline__ int morton_key(double xv, double yv, const Frame &f) {
    return spread_bits(quantize(xv, f.xmin, f.scale)) |
           (spread_bits(quantize(yv, f.ymin, f.scale)) << 1);
}

__global__ __launch_bounds__(256) void k_key_hist(const double *__restrict__ x,
                                                  const double *__restrict__ y, int n,
                                                  const Frame *__restrict__ frame, int npasses,
                                                  int *__restrict__ hist) {
    pdl_begin();
    __shared__ int s[RS_MAX_PASSES + 1][RS_RADIX];
    for (int i = threadIdx.x; i < (RS_MAX_PASSES + 1) * RS_RADIX; i += blockDim.x)
        (&s[0][0])[i] = 0;
    __syncthreads();
    const Frame f = *frame;
    auto count = [&](double xv, double yv) {
        const unsigned k = (unsigned)morton_key(xv, yv, f);
        for (int p = 0; p < npasses; ++p) atomicAdd(&s[p][(k >> (8 * p)) & 0xFF], 1);
        atomicAdd(&s[RS_MAX_PASSES][k >> BUCKET_SHIFT], 1);
    };
    const int gid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0) {
        const double2 *x2 = reinterpret_cast<const double2 *>(x);
        const double2 *y2 = reinterpret_cast<const double2 *>(y);
        for (int i = gid; i < n / 2; i += stride) {
            const double2 a = x2[i], b = y2[i];
            count(a.x, b.x);
            count(a.y, b.y);
        }
        if ((n & 1) && gid == 0) count(x[n - 1], y[n - 1]);
    } else {
        for (int i = gid; i < n; i += stride) count(x[i], y[i]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < (RS_MAX_PASSES + 1) * RS_RADIX; i += blockDim.x) {
        const int c = (&s[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// One 32-byte store of four doubles (st.global.v4.f64; `p` 32-byte aligned).
__device__ __forceinline__ void st_global_v4(double2 *p, double a, double b, double c, double d) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a), "d"(b), "d"(c),
                 "d"(d)
                 : "memory");
}

// The first pass's inputs: the resident sources, the frame, and where records go.
struct FirstPass {
    const double *x, *y, *v;
    const Frame *frame;
    double2 *rec;               // 2 per source: (x, y), (v, index as bits)
    const int *bucket_off;      // exclusive scan of the bucket histogram
    int *bucket_fill;           // slots claimed per bucket so far (zeroed per sort)
};

// One onesweep pass over 8-byte items, digit (item >> shift) & 0xFF: tiles of 3072 items
// (256 threads x 12, four CTAs per SM); the tile's digit counts, then the global digit offsets
// by decoupled look-back, then the stable rank within each warp from digit ballots; items are
// placed in sorted order in shared memory and written out in runs of equal digits.
// `stall_tile` (a test setting, -1 otherwise) names a tile that publishes into `sink` instead
// of its status words, so that the tiles after it wait until `spin_limit` and report
// DEVERR_SPIN_LIMIT.
constexpr int PS_THREADS = 256;
constexpr int PS_WARPS = PS_THREADS / 32;
constexpr int PS_ITEMS = 12;
constexpr int PS_TILE = PS_THREADS * PS_ITEMS;

// FIRST: the first pass of resident values (the tile's items formed from x, y, v, records
// written to their buckets, see FirstPass); otherwise the items are read from `in`.  STALL:
// the instance that honours stall_tile (the test setting; the others ignore it).
template <bool FIRST, bool STALL = false>
__global__ __launch_bounds__(PS_THREADS, FIRST ? 3 : 4) void k_onesweep_items(
    const unsigned long long *__restrict__ in, unsigned long long *__restrict__ out, int n,
    int shift, const int *__restrict__ digit_offsets, unsigned *status, int *tile_counter,
    unsigned *err, int spin_limit, int stall_tile, unsigned *sink, FirstPass fp) {
    pdl_begin();
    __shared__ unsigned long long s_items[PS_TILE];
    __shared__ int s_whist[PS_WARPS][RS_RADIX];
    __shared__ int s_count[RS_RADIX];
    __shared__ int s_tile_start[RS_RADIX];
    __shared__ int s_global[RS_RADIX];
    __shared__ int s_tile;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1);
    for (int i = tid; i < PS_WARPS * RS_RADIX; i += PS_THREADS) (&s_whist[0][0])[i] = 0;
    s_count[tid] = 0;
    if (FIRST) s_global[tid] = 0;   // the tile's count per bucket, first
    __syncthreads();
    const int tile = s_tile;
    const int tile_base = tile * PS_TILE;
    const int tile_n = min(PS_TILE, n - tile_base);
    const int warp_base = tile_base + warp * (PS_ITEMS * 32);

    unsigned long long item[PS_ITEMS];
    int rank[PS_ITEMS];
    if constexpr (FIRST) {
        // keys and each source's slot among the tile's sources of its bucket; the loads are
        // issued in batches of FB before the shared atomics that consume them
        const Frame f = *fp.frame;
        constexpr int FB = 4;
        static_assert(PS_ITEMS % FB == 0, "whole batches");
#pragma unroll
        for (int k0 = 0; k0 < PS_ITEMS; k0 += FB) {
            double xv[FB], yv[FB];
#pragma unroll
            for (int k = 0; k < FB; ++k) {
                const int idx = warp_base + (k0 + k) * 32 + lane;
                xv[k] = idx < n ? __ldg(fp.x + idx) : 0.0;
                yv[k] = idx < n ? __ldg(fp.y + idx) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < FB; ++k) {
                const int idx = warp_base + (k0 + k) * 32 + lane;
                int key = 0, slot = 0;
                if (idx < n) {
                    key = morton_key(xv[k], yv[k], f);
                    slot = atomicAdd(&s_global[(unsigned)key >> BUCKET_SHIFT], 1);
                }
                item[k0 + k] = ((unsigned long long)(unsigned)key << 32) | (unsigned)slot;
            }
        }
        __syncthreads();
        // the tile's slots in each bucket, one global claim per bucket
        {
            const int c = s_global[tid];
            if (c) s_tile_start[tid] = fp.bucket_off[tid] + atomicAdd(&fp.bucket_fill[tid], c);
        }
        __syncthreads();
        // each record with one 32-byte store (one whole DRAM sector), batches of FB loads first
#pragma unroll
        for (int k0 = 0; k0 < PS_ITEMS; k0 += FB) {
            double xv[FB], yv[FB], vv[FB];
#pragma unroll
            for (int k = 0; k < FB; ++k) {
                const int idx = warp_base + (k0 + k) * 32 + lane;
                xv[k] = idx < n ? __ldg(fp.x + idx) : 0.0;
                yv[k] = idx < n ? __ldg(fp.y + idx) : 0.0;
                vv[k] = idx < n ? __ldg(fp.v + idx) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < FB; ++k) {
                const int idx = warp_base + (k0 + k) * 32 + lane;
                if (idx >= n) continue;
                const unsigned key = (unsigned)(item[k0 + k] >> 32);
                const int pos = s_tile_start[key >> BUCKET_SHIFT] + (int)(unsigned)item[k0 + k];
                if ((unsigned)pos >= (unsigned)n) {
                    atomicOr(err, DEVERR_BOUNDS);
                    continue;
                }
                st_global_v4(fp.rec + 2 * (size_t)pos, xv[k], yv[k], vv[k],
                             __longlong_as_double((long long)idx));
                item[k0 + k] = ((unsigned long long)key << 32) | (unsigned)pos;
            }
        }
        __syncthreads();   // s_tile_start is reused below
    } else {
#pragma unroll
        for (int k = 0; k < PS_ITEMS; ++k) {
            const int idx = warp_base + k * 32 + lane;
            item[k] = idx < n ? in[idx] : 0ull;
        }
    }
    // Early counts: the tile's digit totals first (shared atomics), so that its aggregate is
    // published and the look-back done before the ranking, not after it.
    const int d = tid;   // one digit per thread
#pragma unroll
    for (int k = 0; k < PS_ITEMS; ++k)
        if (warp_base + k * 32 + lane < n) atomicAdd(&s_count[(int)(item[k] >> shift) & 0xFF], 1);
    __syncthreads();
    const int total = s_count[d];
    // tile == stall_tile (a test setting): this tile publishes into `sink`, which no look-back
    // reads, so the tiles after it wait until spin_limit
    unsigned *mine = (STALL && tile == stall_tile ? sink : status + (size_t)tile * RS_RADIX) + d;
    int excl = 0;
    if (tile == 0) {
        atomicExch(mine, RS_FLAG_INC | (unsigned)total);
    } else {
        atomicExch(mine, RS_FLAG_AGG | (unsigned)total);
        excl = lookback(status, tile, d, err, spin_limit);
        atomicExch(mine, RS_FLAG_INC | (unsigned)(excl + total));
    }

    const unsigned lt = lanemask_lt();
    int *hist = s_whist[warp];
#pragma unroll
    for (int k = 0; k < PS_ITEMS; ++k) {
        const int idx = warp_base + k * 32 + lane;
        const bool valid = idx < n;
        const unsigned vmask = __ballot_sync(FULL_MASK, valid);
        const int dk = (int)(item[k] >> shift) & 0xFF;
        unsigned peers = digit_peers(vmask, dk);
        if (!valid) peers = 0;
        const int old = valid ? hist[dk] : 0;
        __syncwarp();
        if (valid && (peers & lt) == 0) hist[dk] = old + __popc(peers);
        __syncwarp();
        rank[k] = old + __popc(peers & lt);
    }
    __syncthreads();
    int run = 0;
#pragma unroll
    for (int w = 0; w < PS_WARPS; ++w) {
        const int c = s_whist[w][d];
        s_whist[w][d] = run;
        run += c;
    }
    const int start = block_exclusive_scan(total, nullptr);
    s_tile_start[d] = start;
    s_global[d] = digit_offsets[d] + excl - start;
    __syncthreads();

#pragma unroll
    for (int k = 0; k < PS_ITEMS; ++k) {
        const int idx = warp_base + k * 32 + lane;
        if (idx < n) {
            const int dk = (int)(item[k] >> shift) & 0xFF;
            const int p = s_tile_start[dk] + s_whist[warp][dk] + rank[k];
            if ((unsigned)p >= (unsigned)tile_n) {
                atomicOr(err, DEVERR_BOUNDS);
                continue;
            }
            s_items[p] = item[k];
        }
    }
    __syncthreads();

#pragma unroll 4
    for (int j = tid; j < tile_n; j += PS_THREADS) {
        const unsigned long long it = s_items[j];
        const int g = s_global[(int)(it >> shift) & 0xFF] + j;
        if ((unsigned)g >= (unsigned)n) {
            atomicOr(err, DEVERR_BOUNDS);
            continue;
        }
        out[g] = it;
    }
}

// Sorted keys, permutation, x, y and v from the sorted items and the input-order records.
constexpr int GS_THREADS = 256;
constexpr int GS_ITEMS = 8;

// The sorted sources from the sorted items (key << 32 | record slot) and the bucketed records
// (x, y, v, index): the sorted keys, the permutation (the records' indices) and x, y, v.
__global__ __launch_bounds__(GS_THREADS) void k_gather_sources(
    const unsigned long long *__restrict__ items, const double2 *__restrict__ rec, int n,
    int *__restrict__ keys, int *__restrict__ perm, double *__restrict__ xs,
    double *__restrict__ ys, double *__restrict__ vs, unsigned *err) {
    pdl_begin();
    const int stride = gridDim.x * GS_THREADS * GS_ITEMS;
    for (int base = blockIdx.x * GS_THREADS * GS_ITEMS + threadIdx.x; base < n; base += stride) {
        unsigned long long it[GS_ITEMS];
        double2 a[GS_ITEMS], b[GS_ITEMS];
#pragma unroll
        for (int k = 0; k < GS_ITEMS; ++k) {
            const int i = base + k * GS_THREADS;
            it[k] = i < n ? items[i] : 0ull;
        }
#pragma unroll
        for (int k = 0; k < GS_ITEMS; ++k) {
            const int i = base + k * GS_THREADS;
            const unsigned id = (unsigned)it[k];
            if (i < n && id < (unsigned)n) {
                a[k] = __ldg(rec + 2 * (size_t)id);
                b[k] = __ldg(rec + 2 * (size_t)id + 1);
            }
        }
#pragma unroll
        for (int k = 0; k < GS_ITEMS; ++k) {
            const int i = base + k * GS_THREADS;
            if (i >= n) continue;
            if ((unsigned)it[k] >= (unsigned)n) {
                atomicOr(err, DEVERR_BOUNDS);
                continue;
            }
            keys[i] = (int)(it[k] >> 32);
            perm[i] = (int)__double_as_longlong(b[k].y);
            xs[i] = a[k].x;
            ys[i] = a[k].y;
            vs[i] = b[k].x;
        }
    }
}

// Late values, before they arrive: x and y in sorted order, gathered by the permutation from
// the input arrays (off the critical path, while v is still being copied in).
__global__ __launch_bounds__(256) void k_gather_xy(const int *__restrict__ perm,
                                                   const double *__restrict__ x,
                                                   const double *__restrict__ y, int n,
                                                   double *__restrict__ xs,
                                                   double *__restrict__ ys, unsigned *err) {
    pdl_begin();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned j = (unsigned)perm[i];
        if (j >= (unsigned)n) {
            atomicOr(err, DEVERR_BOUNDS);
            continue;
        }
        xs[i] = __ldg(x + j);
        ys[i] = __ldg(y + j);
    }
}

// Late values, once they are in: v in sorted order (the one gather left after their arrival).
__global__ __launch_bounds__(256) void k_gather_v(const int *__restrict__ perm,
                                                  const double *__restrict__ v, int n,
                                                  double *__restrict__ vs) {
    pdl_begin();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned j = (unsigned)perm[i];
        if (j < (unsigned)n) vs[i] = __ldg(v + j);
    }
}

// Sorted keys and permutation from the sorted items.
__global__ __launch_bounds__(256) void k_items_split(const unsigned long long *__restrict__ items,
                                                     int n, int *__restrict__ keys,
                                                     int *__restrict__ perm) {
    pdl_begin();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long it = items[i];
        keys[i] = (int)(it >> 32);
        perm[i] = (int)(unsigned)it;
    }
}

// The allocation-free sort's gather: the sorted items sit in xs (as 8-byte words); each thread
// reads item i and then overwrites xs[i] with the source's x, so no other buffer is needed.
__global__ __launch_bounds__(256) void k_gather_items_inplace(
    const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ v, int n,
    int *__restrict__ keys, int *__restrict__ perm, double *xs, double *__restrict__ ys,
    double *__restrict__ vs, unsigned *err) {
    unsigned long long *items = reinterpret_cast<unsigned long long *>(xs);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long it = items[i];
        const unsigned j = (unsigned)it;
        if (j >= (unsigned)n) {
            atomicOr(err, DEVERR_BOUNDS);
            continue;
        }
        keys[i] = (int)(it >> 32);
        perm[i] = (int)j;
        xs[i] = x[j];
        ys[i] = y[j];
        vs[i] = v[j];
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
    const bool ovl = c.launch_overlap;   // launch_pdl chains (tc_set_launch_overlap)
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
    // the kernels after k_hist follow each other directly (launch_pdl)
    TC_CUDA_TRY(launch_pdl(ovl, k_hist_scan, npasses, RS_RADIX, 0, c.stream, (const int *)hist,
                           offsets));
    TC_KERNEL_CHECK();
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);

    const int *ki = keys_in, *vi = vals_in;
    int *ko = keys_a, *vo = vals_a;
    for (int p = 0; p < npasses; ++p) {
        TC_CUDA_TRY(launch_pdl(ovl, k_onesweep, ntiles, RS_THREADS, 0, c.stream, ki, vi, ko, vo, n,
                               8 * p, (const int *)(offsets + p * RS_RADIX),
                               status + (size_t)p * ntiles * RS_RADIX, counter + p, err));
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
    pdl_begin();
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
    pdl_begin();
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
    pdl_begin();
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
    const bool ovl = c.launch_overlap;   // launch_pdl chains (tc_set_launch_overlap)
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
    TC_CUDA_TRY(launch_pdl(ovl, k_scan_blocks, 1, SCAN_THREADS, 0, c.stream, bs, nb, d_out + n));
    TC_KERNEL_CHECK();
    TC_CUDA_TRY(launch_pdl(ovl, k_scan_apply, nb, SCAN_THREADS, 0, c.stream, d_in, n,
                           (const int *)bs, d_out));
    TC_KERNEL_CHECK();
    return TC_OK;
}

// ---------------------------------------------------------------------------- drivers
int sort_sources(Context &c, const double *x, const double *y, const double *v, int n,
                 cudaEvent_t values_ready) {
    const bool ovl = c.launch_overlap;   // launch_pdl chains (tc_set_launch_overlap)
    int rc;
    c.late_ready = nullptr;   // a late-value sort of an earlier call that failed midway
    double *xs, *ys, *vs;
    int *keys, *perm;
    Frame *frame;
    double4 *partials;
    if ((rc = ensure(c, S_XS, n, &xs)) || (rc = ensure(c, S_YS, n, &ys)) ||
        (rc = ensure(c, S_VS, n, &vs)) || (rc = ensure(c, S_KEYS, n, &keys)) ||
        (rc = ensure(c, S_PERM, n, &perm)))
        return rc;
    // frame + bbox partials + completion counter share one small buffer
    const int gb = grid_for(n, BBOX_THREADS, 8);
    if ((rc = ensure(c, S_FRAME, sizeof(Frame) + sizeof(double4) * (gb + 1) + 64, (char **)&frame)))
        return rc;
    partials = reinterpret_cast<double4 *>(reinterpret_cast<char *>(frame) + 64);
    unsigned *done = reinterpret_cast<unsigned *>(partials + gb);

    // four 8-bit passes over the (key, index) items, then one gather of the records
    if (n >= (1 << 30)) {
        set_error(TC_ERR_INVALID, "too many sources for the radix sort (%d)", n);
        return TC_ERR_INVALID;
    }
    unsigned long long *items_a, *items_b;
    double2 *rec;
    int *hist, *counter;
    unsigned *status;
    const int npasses = (2 * LMAX + 7) / 8;
    const int ntiles = (n + PS_TILE - 1) / PS_TILE;
    // histograms and their scans: the four radix digits, then the buckets of the records
    constexpr int NHIST = RS_MAX_PASSES + 1;
    if ((rc = ensure(c, S_ITEMS_A, n, &items_a)) || (rc = ensure(c, S_ITEMS_B, n, &items_b)) ||
        (rc = ensure(c, S_REC, 2 * (size_t)n, &rec)) ||
        (rc = ensure(c, S_RS_HIST, 2 * NHIST * RS_RADIX, &hist)) ||
        (rc = ensure(c, S_RS_COUNTER, RS_MAX_PASSES + NB_BUCKETS, &counter)) ||
        (rc = ensure(c, S_RS_STATUS, ((size_t)RS_MAX_PASSES * ntiles + 1) * RS_RADIX, &status)))
        return rc;
    int *offsets = hist + NHIST * RS_RADIX;
    unsigned *sink = status + (size_t)RS_MAX_PASSES * ntiles * RS_RADIX;   // after every pass
    int *bucket_fill = counter + RS_MAX_PASSES;
    // every buffer and counter first, so that the sort's kernels follow each other directly on
    // the stream (each may then be scheduled while the one before it drains, launch_pdl)
    TC_CUDA_TRY(cudaMemsetAsync(done, 0, sizeof(unsigned), c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(int) * NHIST * RS_RADIX, c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int) * (RS_MAX_PASSES + NB_BUCKETS), c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned) * (size_t)npasses * ntiles * RS_RADIX,
                                c.stream));
    k_bbox<<<gb, BBOX_THREADS, 0, c.stream>>>(x, y, n, partials, done, frame);
    TC_KERNEL_CHECK();
    // resident values: the records are written by the first pass, in buckets (see FirstPass);
    // values that arrive later: items in input order; x, y, v gathered by the permutation
    // in finish_sources
    const bool bucketed = values_ready == nullptr;
    if (bucketed)
        TC_CUDA_TRY(launch_pdl(ovl, k_key_hist, grid_for(n, 256, 8), 256, 0, c.stream, x, y, n,
                               (const Frame *)frame, npasses, hist));
    else
        TC_CUDA_TRY(launch_pdl(ovl, k_keys_pack, grid_for(n, 256, 8), 256, 0, c.stream, x, y, n,
                               (const Frame *)frame, items_a, npasses, hist));
    TC_KERNEL_CHECK();
    TC_CUDA_TRY(launch_pdl(ovl, k_hist_scan, NHIST, RS_RADIX, 0, c.stream, (const int *)hist,
                           offsets));
    TC_KERNEL_CHECK();
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);
    const FirstPass fp = {x, y, v, frame, rec, offsets + RS_MAX_PASSES * RS_RADIX, bucket_fill};
    static_assert((2 * LMAX + 7) / 8 % 2 == 0, "an even number of passes ends in items_a");
    for (int p = 0; p < npasses; ++p) {
        const bool odd = p & 1;
        const int stall = p == 0 && c.test_stall == TC_STALL_SORT ? 0 : -1;
        auto pass = p == 0 ? (bucketed ? (stall >= 0 ? k_onesweep_items<true, true>
                                                   : k_onesweep_items<true, false>)
                                       : (stall >= 0 ? k_onesweep_items<false, true>
                                                     : k_onesweep_items<false, false>))
                           : k_onesweep_items<false, false>;
        TC_CUDA_TRY(launch_pdl(ovl, pass, ntiles, PS_THREADS, 0, c.stream,
                               (const unsigned long long *)(odd ? items_b : items_a),
                               odd ? items_a : items_b, n, 32 + 8 * p,
                               (const int *)(offsets + p * RS_RADIX),
                               status + (size_t)p * ntiles * RS_RADIX, counter + p, err,
                               c.spin_limit, stall, sink, fp));
        TC_KERNEL_CHECK();
    }
    c.nsrc = n;
    // a test stall leaves the passes' output unordered: report it before anything reads it
    if (c.test_stall == TC_STALL_SORT && (rc = check_device_errors(c, "source sort"))) return rc;
    if (values_ready) {
        // the keys now (the tree needs nothing else); x, y, v in finish_sources
        TC_CUDA_TRY(launch_pdl(ovl, k_items_split, grid_for(n, 256, 8), 256, 0, c.stream,
                               (const unsigned long long *)items_a, n, keys, perm));
        TC_KERNEL_CHECK();
        c.late_x = x;
        c.late_y = y;
        c.late_v = v;
        c.late_ready = values_ready;
        return TC_OK;
    }
    // a window of the sorted order in flight at a time (4 CTAs per SM): its records come from
    // a compact range of buckets, which stays in L2
    TC_CUDA_TRY(launch_pdl(ovl, k_gather_sources, grid_for(n, GS_THREADS * GS_ITEMS, 4),
                           GS_THREADS, 0, c.stream, (const unsigned long long *)items_a,
                           (const double2 *)rec, n, keys, perm, xs, ys, vs, err));
    TC_KERNEL_CHECK();
    return TC_OK;
}

int finish_sources(Context &c) {
    if (!c.late_ready) return TC_OK;
    const int n = c.nsrc;
    const int *perm = slot_ptr<int>(c, S_PERM);
    k_gather_xy<<<grid_for(n, 256, 8), 256, 0, c.stream>>>(perm, c.late_x, c.late_y, n,
                                                          slot_ptr<double>(c, S_XS),
                                                          slot_ptr<double>(c, S_YS),
                                                          slot_ptr<unsigned>(c, S_ERR));
    TC_KERNEL_CHECK();
    TC_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.late_ready, 0));
    c.late_ready = nullptr;
    k_gather_v<<<grid_for(n, 256, 8), 256, 0, c.stream>>>(perm, c.late_v, n,
                                                         slot_ptr<double>(c, S_VS));
    TC_KERNEL_CHECK();
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
// Source sort for callers that cannot allocate device memory, on the kernels the host entry
// points run (k_bbox, k_keys_pack, four k_onesweep_items passes).  The caller's output arrays
// double as the passes' ping-pong buffers: the 8-byte items live in xsorted and ysorted until
// the last pass, and the gather then overwrites them in place.  Everything else -- the
// per-tile look-back words, the digit histograms and their scans, the tile counters, the
// bounding-box partials and the error word -- lives in one static device array of fixed size,
// so a call makes no cudaMalloc/cudaFree and no other allocating call.
constexpr int NOALLOC_MAX_SOURCES = 1 << 20;
constexpr int NA_MAX_TILES = (NOALLOC_MAX_SOURCES + PS_TILE - 1) / PS_TILE;
constexpr int NA_MAX_BBOX_BLOCKS = 4096;
constexpr size_t NA_OFF_STATUS = 0;
constexpr size_t NA_OFF_HIST =
    NA_OFF_STATUS + sizeof(unsigned) * RS_MAX_PASSES * NA_MAX_TILES * RS_RADIX;
constexpr size_t NA_OFF_CTR = NA_OFF_HIST + sizeof(int) * 2 * RS_MAX_PASSES * RS_RADIX;
constexpr size_t NA_OFF_ERR = NA_OFF_CTR + 256;
constexpr size_t NA_OFF_DONE = NA_OFF_ERR + 256;
constexpr size_t NA_OFF_PARTIALS = NA_OFF_DONE + 256;
constexpr size_t NA_BYTES = NA_OFF_PARTIALS + sizeof(double4) * NA_MAX_BBOX_BLOCKS;  // ~1.5 MB

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

void kernels_sort(KernelList &v) {
    v.insert(v.end(), {(const void *)k_bbox, (const void *)k_target_keys,
                       (const void *)k_gather_items_inplace, (const void *)k_hist,
                       (const void *)k_hist_scan,
                       (const void *)k_onesweep, (const void *)k_keys_pack,
                       (const void *)k_onesweep_items<true>,
                       (const void *)k_onesweep_items<false>, (const void *)k_key_hist,
                       (const void *)k_onesweep_items<true, true>,
                       (const void *)k_onesweep_items<false, true>,
                       (const void *)k_gather_sources, (const void *)k_gather_xy,
                       (const void *)k_gather_v, (const void *)k_items_split,
                       (const void *)k_scan_reduce, (const void *)k_scan_blocks,
                       (const void *)k_scan_apply});
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
    unsigned *status = reinterpret_cast<unsigned *>(base + NA_OFF_STATUS);
    int *hist = reinterpret_cast<int *>(base + NA_OFF_HIST);
    int *offsets = hist + RS_MAX_PASSES * RS_RADIX;
    int *counter = reinterpret_cast<int *>(base + NA_OFF_CTR);
    unsigned *err = reinterpret_cast<unsigned *>(base + NA_OFF_ERR);
    unsigned *done = reinterpret_cast<unsigned *>(base + NA_OFF_DONE);
    double4 *partials = reinterpret_cast<double4 *>(base + NA_OFF_PARTIALS);
    Frame *fr = reinterpret_cast<Frame *>(frame);
    // the passes' ping-pong buffers: the caller's xsorted / ysorted, as 8-byte items
    unsigned long long *items_a = reinterpret_cast<unsigned long long *>(xsorted);
    unsigned long long *items_b = reinterpret_cast<unsigned long long *>(ysorted);

    // The array keeps the previous call's contents: clear what has to start at zero.
    const int npasses = (2 * LMAX + 7) / 8;
    const int ntiles = (n + PS_TILE - 1) / PS_TILE;
    TC_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(unsigned), s));
    TC_CUDA_TRY(cudaMemsetAsync(done, 0, sizeof(unsigned), s));
    TC_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(int) * RS_MAX_PASSES * RS_RADIX, s));
    TC_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int) * RS_MAX_PASSES, s));
    TC_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned) * (size_t)npasses * ntiles * RS_RADIX, s));

    const int gb = std::min(grid_for(n, BBOX_THREADS, 8), NA_MAX_BBOX_BLOCKS);
    k_bbox<<<gb, BBOX_THREADS, 0, s>>>(xsources, ysources, n, partials, done, fr);
    TC_KERNEL_CHECK();
    k_keys_pack<<<grid_for(n, 256, 8), 256, 0, s>>>(xsources, ysources, n, fr, items_a, npasses,
                                                    hist);
    TC_KERNEL_CHECK();
    k_hist_scan<<<npasses, RS_RADIX, 0, s>>>(hist, offsets);
    TC_KERNEL_CHECK();
    static_assert((2 * LMAX + 7) / 8 % 2 == 0, "an even number of passes ends in items_a");
    for (int p = 0; p < npasses; ++p) {
        const bool odd = p & 1;
        k_onesweep_items<false><<<ntiles, PS_THREADS, 0, s>>>(
            odd ? items_b : items_a, odd ? items_a : items_b, n, 32 + 8 * p,
            offsets + p * RS_RADIX, status + (size_t)p * ntiles * RS_RADIX, counter + p, err,
            RS_SPIN_LIMIT, -1, nullptr, FirstPass{});
        TC_KERNEL_CHECK();
    }
    k_gather_items_inplace<<<grid_for(n, 256), 256, 0, s>>>(xsources, ysources, sourcevalues, n,
                                                             keys, perm, xsorted, ysorted,
                                                             vsorted, err);
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
