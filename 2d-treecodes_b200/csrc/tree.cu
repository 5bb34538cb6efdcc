// tree.cu -- quadtree topology from the sorted Morton keys.
//
// Restates the top-down split of drivers/upward.cpp:223-277 without recursion.  A cell at
// level l with key prefix P exists iff its parent is split; it is split ("inner") iff it holds
// more than L sources and l < LMAX (upward.cpp:245).  Both facts can be read off the sorted
// keys at O(1) cost per source:
//   * source i starts the level-l run of its prefix iff keys[i-1] and keys[i] differ at level l;
//   * that run holds more than L sources iff keys[i+L] has the same level-l prefix.
// So each source yields a bit mask of the levels at which it starts an inner cell.  The cells
// are numbered breadth first (level by level, Morton order inside a level, children c = 0..3
// contiguous), the same canonical order in which the tests walk the reference's tree; the
// reference's own numbering depends on OpenMP task timing.  Child ranges come from exact
// binary searches for the child key boundaries, the bounds lower_bound_vec/upper_bound_vec
// (kernels/upward-common.ispc:59-124) compute.
//
// Node arrays (HBM, one entry per node, breadth-first order):
//   TNode tnode    {xcom, ycom, r, child, count}  32 B   (traversal record)
//   int2  range    {s, e}                           8 B
//   int4  cell     {level, cx, cy, parent}         16 B
#include "tc_internal.h"

namespace tc {

// Largest level at which the prefixes of two keys agree (0..LMAX).
__device__ __forceinline__ int common_level(int a, int b) {
    const unsigned x = (unsigned)(a ^ b);
    if (!x) return LMAX;
    const int hb = 31 - __clz(x);
    return LMAX - 1 - hb / 2;
}

__device__ __forceinline__ int lower_bound_dev(const int *__restrict__ keys, int lo, int hi,
                                               int val) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (keys[mid] < val) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// The same bound, found by doubling steps from lo first: O(log(answer - lo)) reads, which is
// what pays for the many small cells of the deep levels.
__device__ __forceinline__ int gallop_lower_bound(const int *__restrict__ keys, int lo, int hi,
                                                  int val) {
    if (lo >= hi || keys[lo] >= val) return lo;
    int a = lo, step = 1;   // keys[a] < val
    while (a + step < hi && keys[a + step] < val) {
        a += step;
        step <<= 1;
    }
    return lower_bound_dev(keys, a + 1, min(a + step, hi), val);
}

// The split list: per tile of TL_TILE sources, each source's level mask (bit l: it starts an
// inner cell of level l), a block scan
// of the flags and the tile's global offset by a decoupled look-back over the tiles before it
// (tile ids from an atomic counter, so a tile only waits on tiles already running; one warp
// reads 32 predecessors per step; the wait is bounded and raises DEVERR_SPIN_LIMIT).  The tile
// that holds the last source writes the list length to *nlist_out.
constexpr int TL_THREADS = 256;
constexpr int TL_ITEMS = 16;
constexpr int TL_TILE = TL_THREADS * TL_ITEMS;
constexpr int TL_HALO = LEAF_POTENTIAL;           // the largest leaf capacity
constexpr int TL_STAGE = TL_TILE + 1 + TL_HALO;   // staged keys per tile
constexpr unsigned TL_AGG = 1u << 30, TL_INC = 2u << 30, TL_VAL = (1u << 30) - 1;
// `stall_tile` (a test setting, -1 otherwise) names a tile that publishes nothing, so that the
// tile after it waits until `spin_limit` and reports DEVERR_SPIN_LIMIT.

__global__ __launch_bounds__(TL_THREADS) void k_tree_list(const int *__restrict__ keys, int n,
                                                          int leafcap, int cap, unsigned *status,
                                                          int *tile_counter, int *__restrict__ lpos,
                                                          unsigned short *__restrict__ lmask,
                                                          int *nlist_out, unsigned *err,
                                                          int spin_limit, int stall_tile) {
    pdl_begin();
    __shared__ int s_tile, s_excl;
    // the tile's keys with one before and leafcap after, staged by coalesced loads; word q is
    // kept at q + q / 32 so that the 16-source runs of a warp's threads hit distinct banks
    __shared__ int s_keys[TL_STAGE + TL_STAGE / 32 + 1];
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1);
    __syncthreads();
    const int tile = s_tile;
    const int base = tile * TL_TILE - 1;   // key index of staged word 0
    if (leafcap > TL_HALO) {
        if (threadIdx.x == 0) atomicOr(err, DEVERR_BOUNDS);
        return;   // every thread of every tile takes this branch: nothing waits on it
    }
    const int span = min(TL_TILE + 1 + leafcap, n - base);
    for (int q = threadIdx.x; q < span; q += TL_THREADS) {
        const int i = base + q;
        s_keys[q + (q >> 5)] = i >= 0 ? keys[i] : 0;
    }
    __syncthreads();
    auto staged = [&](int i) {
        const int q = i - base;
        return s_keys[q + (q >> 5)];
    };
    const int i0 = tile * TL_TILE + threadIdx.x * TL_ITEMS;   // this thread's 16 sources
    unsigned short m[TL_ITEMS];
    int cnt = 0;
    int prev = i0 > 0 && i0 <= n ? staged(i0 - 1) : 0;
#pragma unroll
    for (int k = 0; k < TL_ITEMS; ++k) {
        const int i = i0 + k;
        unsigned mk = 0;
        if (i < n) {
            const int key = staged(i);
            const int cprev = i == 0 ? -1 : common_level(prev, key);
            const int cnext = i + leafcap < n ? common_level(key, staged(i + leafcap)) : -1;
            const int hi = min(cnext, LMAX - 1);
            for (int l = cprev + 1; l <= hi; ++l) mk |= 1u << l;
            prev = key;
        }
        m[k] = (unsigned short)mk;
        cnt += mk != 0;
    }
    int total;
    const int toff = block_exclusive_scan(cnt, &total);
    // Look-back by warp 0: 32 predecessors per step, lane q reading tile - 1 - q - (consumed)
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        unsigned *mine = status + tile;
        const bool publish = tile != stall_tile;
        int excl = 0;
        if (tile == 0) {
            if (lane == 0 && publish) atomicExch(mine, TL_INC | (unsigned)total);
        } else {
            if (lane == 0 && publish) atomicExch(mine, TL_AGG | (unsigned)total);
            int j = tile - 1, spins = 0;
            for (;;) {
                const int jj = j - lane;
                // before tile 0 reads as an inclusive prefix of 0
                const unsigned st = jj >= 0 ? *(const volatile unsigned *)(status + jj) : TL_INC;
                const unsigned flag = st & ~TL_VAL;
                const unsigned inc = __ballot_sync(FULL_MASK, flag == TL_INC);
                const unsigned none = __ballot_sync(FULL_MASK, flag == 0);
                const int first_inc = inc ? __ffs(inc) - 1 : 31;
                const unsigned upto = (2u << first_inc) - 1u;   // lanes 0 .. first_inc
                if (none & upto) {
                    // add what is published before the first unpublished predecessor, then
                    // read again from it
                    const int first_none = __ffs(none & upto) - 1;
                    excl += __reduce_add_sync(FULL_MASK, lane < first_none ? st & TL_VAL : 0u);
                    j -= first_none;
                    if (first_none == 0 && ++spins > spin_limit) {
                        if (lane == 0) atomicOr(err, DEVERR_SPIN_LIMIT);
                        break;
                    }
                    continue;
                }
                excl += __reduce_add_sync(FULL_MASK, lane <= first_inc ? st & TL_VAL : 0u);
                if (inc) break;
                j -= 32;
            }
            if (lane == 0 && publish) atomicExch(mine, TL_INC | (unsigned)(excl + total));
        }
        if (lane == 0) {
            s_excl = excl;
            if ((long long)(tile + 1) * TL_TILE >= n) *nlist_out = excl + total;
        }
    }
    __syncthreads();
    int j = s_excl + toff;
#pragma unroll
    for (int k = 0; k < TL_ITEMS; ++k)
        if (m[k]) {
            if (j < cap) {
                lpos[j] = i0 + k;
                lmask[j] = m[k];
            } else {
                atomicOr(err, DEVERR_TREE);
            }
            ++j;
        }
}

constexpr int RANK_THREADS = 1024;

// Per block of 1024 list entries: how many have bit l, for every level l.
__global__ __launch_bounds__(RANK_THREADS) void k_rank_count(const unsigned short *__restrict__ lmask,
                                                             const int *__restrict__ d_nlist,
                                                             int *__restrict__ blk, int nblk) {
    pdl_begin();
    __shared__ int s_cnt[LMAX];
    if (threadIdx.x < LMAX) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    const int nlist = *d_nlist;
    const int j = blockIdx.x * RANK_THREADS + threadIdx.x;
    const unsigned m = j < nlist ? lmask[j] : 0u;
    for (int l = 0; l < LMAX; ++l) {
        const unsigned b = __ballot_sync(FULL_MASK, (m >> l) & 1u);
        if (lane_id() == 0 && b) atomicAdd(&s_cnt[l], __popc(b));
    }
    __syncthreads();
    if (threadIdx.x < LMAX) blk[threadIdx.x * nblk + blockIdx.x] = s_cnt[threadIdx.x];
}

// One CTA per level: exclusive scan over the blocks' counts; level total -> totals[l].
__global__ __launch_bounds__(1024) void k_rank_scan(int *__restrict__ blk, int nblk,
                                                    int *__restrict__ totals) {
    pdl_begin();
    __shared__ int s_part[1024];
    const int l = blockIdx.x;
    int *row = blk + (size_t)l * nblk;
    const int per = (nblk + 1023) / 1024;
    const int b0 = threadIdx.x * per;
    int s = 0;
    for (int i = 0; i < per; ++i)
        if (b0 + i < nblk) s += row[b0 + i];
    s_part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int t = 0; t < 1024; ++t) {
            const int v = s_part[t];
            s_part[t] = run;
            run += v;
        }
        totals[l] = run;
    }
    __syncthreads();
    int run = s_part[threadIdx.x];
    for (int i = 0; i < per; ++i)
        if (b0 + i < nblk) {
            const int v = row[b0 + i];
            row[b0 + i] = run;
            run += v;
        }
}

// rank[l * stride + j] = number of list entries before j that have bit l (for every entry j,
// with or without bit l).
// inv[l * stride + r] = the entry whose level-l inner cell has rank r.
__global__ __launch_bounds__(RANK_THREADS) void k_rank_apply(const unsigned short *__restrict__ lmask,
                                                             const int *__restrict__ d_nlist,
                                                             const int *__restrict__ blk, int nblk,
                                                             int *__restrict__ rank,
                                                             int *__restrict__ inv, int stride) {
    pdl_begin();
    __shared__ int s_w[LMAX][RANK_THREADS / 32];
    const int nlist = *d_nlist;
    const int j = blockIdx.x * RANK_THREADS + threadIdx.x;
    const int w = threadIdx.x >> 5;
    const unsigned m = j < nlist ? lmask[j] : 0u;
    unsigned bal[LMAX];
#pragma unroll
    for (int l = 0; l < LMAX; ++l) {
        bal[l] = __ballot_sync(FULL_MASK, (m >> l) & 1u);
        if (lane_id() == 0) s_w[l][w] = __popc(bal[l]);
    }
    __syncthreads();
    if (threadIdx.x < LMAX) {
        int run = 0;
        for (int t = 0; t < RANK_THREADS / 32; ++t) {
            const int v = s_w[threadIdx.x][t];
            s_w[threadIdx.x][t] = run;
            run += v;
        }
    }
    __syncthreads();
    if (j < nlist) {
        const unsigned lt = lanemask_lt();
#pragma unroll
        for (int l = 0; l < LMAX; ++l) {
            const int r = blk[(size_t)l * nblk + blockIdx.x] + s_w[l][w] + __popc(bal[l] & lt);
            rank[(size_t)l * stride + j] = r;
            if ((m >> l) & 1u) inv[(size_t)l * stride + r] = j;
        }
    }
}


__global__ void k_tree_root(int n, int leafcap, TNode *tnode, int2 *range, int4 *cell) {
    pdl_begin();
    range[0] = make_int2(0, n);
    cell[0] = make_int4(0, 0, 0, -1);
    tnode[0].count = n;
    if (n <= leafcap) tnode[0].child = -1;
}

// Four threads per inner cell: the r-th inner cell of level l is started by list entry
// inv[l][r] (source s = lpos[j]); its own id comes from its parent's rank.  Thread q of the four
// finds the end of child q (the key boundary of child q + 1, or of the cell's end for q = 3) by
// a search from s; the four searches run at once instead of one after another (each boundary
// lies inside [s, e), since the keys are sorted), and thread q writes child q.
__global__ void k_tree_children(const int *__restrict__ keys, int n, int leafcap,
                                const int *__restrict__ lpos,
                                const unsigned short *__restrict__ lmask,
                                const int *__restrict__ rank, const int *__restrict__ inv,
                                int stride, int ninner, LevelOffsets lo, int nnodes,
                                TNode *__restrict__ tnode, int2 *__restrict__ range,
                                int4 *__restrict__ cell, unsigned *err) {
    pdl_begin();
    const int q = threadIdx.x & 3;
    const unsigned gmask = 0xFu << (lane_id() & ~3);   // the cell's four lanes
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 2; t < ninner;
         t += (gridDim.x * blockDim.x) >> 2) {
        // level of inner cell t: the inner cells are numbered level by level (the four threads
        // compute the same values, so they branch together)
        int l = 0, r = t;
        while (l < LMAX - 1 && r >= (lo.off[l + 2] - lo.off[l + 1]) / 4) {
            r -= (lo.off[l + 2] - lo.off[l + 1]) / 4;
            ++l;
        }
        const int j = inv[(size_t)l * stride + r];
        const int s = lpos[j];
        const unsigned mj = lmask[j];
        if (!((mj >> l) & 1u)) {
            if (q == 0) atomicOr(err, DEVERR_TREE);
            continue;
        }
        const int key = keys[s];
        const int shift = 2 * (LMAX - l);
        const int P = l == 0 ? 0 : (key >> shift);
        int id = 0;
        if (l > 0) {
            // The parent is the inner cell of level l-1 that holds source s: the last list
            // entry up to j with bit l-1 (a later one would start a new level-(l-1) cell
            // before s).  Its rank is the count of such entries up to j, minus one.
            const int prank = rank[(size_t)(l - 1) * stride + j] + (int)((mj >> (l - 1)) & 1u) - 1;
            if (prank < 0) {
                if (q == 0) atomicOr(err, DEVERR_TREE);
                continue;
            }
            id = lo.off[l] + 4 * prank + (P & 3);
        }
        const int base = lo.off[l + 1] + 4 * r;
        if (id < 0 || id >= nnodes || base < 0 || base + 4 > nnodes) {
            if (q == 0) atomicOr(err, DEVERR_BOUNDS);
            continue;
        }
        if (q == 0) tnode[id].child = base;
        const int cshift = shift - 2;
        // the end of child q: the first key of child q + 1, or past the cell for q = 3
        int end_q;
        if (q < 3)
            end_q = gallop_lower_bound(keys, s, n, ((P << 2) | (q + 1)) << cshift);
        else
            end_q = l == 0 ? n : gallop_lower_bound(keys, s, n, (P + 1) << shift);
        int beg_q = __shfl_up_sync(gmask, end_q, 1, 4);
        if (q == 0) beg_q = s;
        const int cx = compact_bits(P), cy = compact_bits(P >> 1);
        const int cid = base + q;
        const int cnt = end_q - beg_q;
        range[cid] = make_int2(beg_q, end_q);
        cell[cid] = make_int4(l + 1, 2 * cx + (q & 1), 2 * cy + (q >> 1), id);
        tnode[cid].count = cnt;
        const bool inner = cnt > leafcap && l + 1 < LMAX;
        if (!inner) tnode[cid].child = -1;
    }
}

static int grid_for_tree(int n, int threads) {
    long long g = ((long long)n + threads - 1) / threads;
    if (g > 148 * 8) g = 148 * 8;
    if (g < 1) g = 1;
    return (int)g;
}

int build_topology(Context &c, int leafcap) {
    const bool ovl = c.launch_overlap;   // launch_pdl chains (tc_set_launch_overlap)
    const int n = c.nsrc;
    int rc;
    const int *keys = slot_ptr<int>(c, S_KEYS);
    // Upper bound of the list length (every inner cell has > leafcap sources in one level):
    // n/(L+1) per level.  The rank arrays are laid out with this stride, so nothing waits for
    // the actual length before the level totals are read back.
    const long long bound = (long long)LMAX * (n / (leafcap + 1) + 1);
    const int cap = (int)(bound < n ? bound : n);
    const int ntl = (n + TL_TILE - 1) / TL_TILE;
    const int nblk = (cap + RANK_THREADS - 1) / RANK_THREADS;
    int *lpos, *rank, *rinv, *blkc, *totals, *tl_counter;
    unsigned *tl_status;
    unsigned short *lmask;
    if ((rc = ensure(c, S_LPOS, (size_t)cap + 1, &lpos)) ||
        (rc = ensure(c, S_LMASK, (size_t)cap + 1, &lmask)) ||
        (rc = ensure(c, S_TFLAG, (size_t)ntl + 8, &tl_status)) ||
        (rc = ensure(c, S_LRANK, (size_t)LMAX * (cap + 1), &rank)) ||
        (rc = ensure(c, S_LINV, (size_t)LMAX * (cap + 1), &rinv)) ||
        (rc = ensure(c, S_LBLK, (size_t)LMAX * (nblk + 1), &blkc)) ||
        (rc = ensure(c, S_LEVEL_TOTALS, LMAX + 4, &totals)))
        return rc;
    int *d_nlist = totals + LMAX;
    tl_counter = totals + LMAX + 1;
    TC_CUDA_TRY(cudaMemsetAsync(totals, 0, sizeof(int) * (LMAX + 4), c.stream));
    TC_CUDA_TRY(cudaMemsetAsync(tl_status, 0, sizeof(unsigned) * ntl, c.stream));
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);
    k_tree_list<<<ntl, TL_THREADS, 0, c.stream>>>(keys, n, leafcap, cap, tl_status, tl_counter,
                                                   lpos, lmask, d_nlist, err, c.spin_limit,
                                                   c.test_stall == TC_STALL_TREE ? 0 : -1);
    TC_KERNEL_CHECK();
    // a test stall leaves the list offsets wrong: report it before anything reads them
    if (c.test_stall == TC_STALL_TREE && (rc = check_device_errors(c, "tree build"))) return rc;
    // the rank kernels follow k_tree_list directly (launch_pdl)
    TC_CUDA_TRY(launch_pdl(ovl, k_rank_count, nblk, RANK_THREADS, 0, c.stream,
                           (const unsigned short *)lmask, (const int *)d_nlist, blkc, nblk));
    TC_KERNEL_CHECK();
    TC_CUDA_TRY(launch_pdl(ovl, k_rank_scan, LMAX, 1024, 0, c.stream, blkc, nblk, totals));
    TC_KERNEL_CHECK();
    TC_CUDA_TRY(launch_pdl(ovl, k_rank_apply, nblk, RANK_THREADS, 0, c.stream,
                           (const unsigned short *)lmask, (const int *)d_nlist, (const int *)blkc,
                           nblk, rank, rinv, cap));
    TC_KERNEL_CHECK();
    // the level totals and the list length, in one read-back
    TC_CUDA_TRY(cudaMemcpyAsync(c.h_pinned, totals, sizeof(int) * (LMAX + 1),
                                cudaMemcpyDeviceToHost, c.stream));
    TC_CUDA_TRY(wait_stream(c, c.stream));
    const int nlist = (int)c.h_pinned[LMAX];
    if (nlist > cap) {
        set_error(TC_ERR_INVALID, "tree list length %d exceeds its bound %d", nlist, cap);
        return TC_ERR_INVALID;
    }
    LevelOffsets lo;
    lo.off[0] = 0;
    lo.off[1] = 1;
    long long ninner = 0;
    int nlevels = 1;
    for (int l = 0; l < LMAX; ++l) {
        const int inner = (int)c.h_pinned[l];
        ninner += inner;
        lo.off[l + 2] = lo.off[l + 1] + 4 * inner;
        if (inner) nlevels = l + 2;
    }
    const long long nnodes = 1 + 4 * ninner;
    if (nnodes >= (1LL << 31)) {
        set_error(TC_ERR_INVALID, "too many tree nodes (%lld)", nnodes);
        return TC_ERR_INVALID;
    }
    c.nnodes = (int)nnodes;
    c.ninner = (int)ninner;
    c.leafcap = leafcap;
    for (int l = 0; l < LMAX + 2; ++l) c.level_off[l] = lo.off[l];
    c.counts.nnodes = nnodes;
    c.counts.ninner = ninner;
    c.counts.nleaves = nnodes - ninner;
    c.counts.nlevels = nlevels;

    TNode *tnode;
    int2 *range;
    int4 *cell;
    if ((rc = ensure(c, S_TNODE, nnodes, &tnode)) || (rc = ensure(c, S_RANGE, nnodes, &range)) ||
        (rc = ensure(c, S_CELL, nnodes, &cell)))
        return rc;
    k_tree_root<<<1, 1, 0, c.stream>>>(n, leafcap, tnode, range, cell);
    TC_KERNEL_CHECK();
    if (ninner > 0) {
        TC_CUDA_TRY(launch_pdl(ovl, k_tree_children, grid_for_tree(4 * (int)ninner, 128), 128, 0,
                               c.stream, keys, n, leafcap, (const int *)lpos,
                               (const unsigned short *)lmask, (const int *)rank,
                               (const int *)rinv, cap, (int)ninner, lo, c.nnodes, tnode, range,
                               cell, slot_ptr<unsigned>(c, S_ERR)));
        TC_KERNEL_CHECK();
    }
    return TC_OK;
}

void kernels_tree(KernelList &v) {
    v.insert(v.end(), {(const void *)k_tree_list, (const void *)k_rank_count,
                       (const void *)k_rank_scan, (const void *)k_rank_apply,
                       (const void *)k_tree_root, (const void *)k_tree_children});
}

}  // namespace tc
