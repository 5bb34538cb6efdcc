// force.cu -- treecode_force_mrag on the GPU: per-brick interaction lists, then the far field
// and the near field of every 8 x 8 brick.
//
// Restates drivers/treecode-force.cpp:94-199 (traversal) and kernels/force-kernels.m4
// (P2P, E2P, E2L, L2P).  An MRAG block of 32 x 32 targets is 16 bricks of 8 x 8
// (treecode-force.cpp:110-111), brick q = (by/8)*4 + bx/8.
//
// 1. k_force_lists<false>: one warp per brick walks the tree 32 nodes at a time and classifies
//    every node with the reference's two criteria (treecode-force.cpp:136-151):
//      E2L  iff  dist(brick centre, com)/r - 1 > 1/theta  and  r_brick <= r
//      E2P  iff  r^2 < theta^2 |clamp(com to brick) - com|^2
//      else P2P for a leaf, descend for an inner node.
//    Counts per brick and kind are compacted with warp ballots.  The arithmetic is the one
//    the compiled reference executes (fma(dx, dx, dy*dy), brick centre fma(bx + 3.5, h, x0),
//    r_brick = 4.949747468305833 h), so every decision is the reference's.
// 2. exclusive scan of the 3 x nbricks counts -> list offsets (E2L | E2P | P2P lists).
// 3. k_force_lists<true>: same walk, writes node ids into the lists.
// 4. k_force_far: persistent warps over bricks, 2 targets per lane; local expansion from the
//    E2L list (lane l owns coefficient l), L2P, E2P from the E2P list, written into the
//    ix + 32*(iy + 32*ib) layout (treecode-force.cpp:191-197).
// 5. k_force_near: persistent warps over tasks, a task being a segment of at most P2P_SEG
//    sources of a brick's P2P list; P2P over the listed leaves with source tiles staged in
//    shared memory.  Single-task bricks add their sums to the outputs; the parts of multi-task
//    bricks are added in task order by k_force_gather_parts, so results are deterministic.
#include <cfloat>

#include "tc_internal.h"
#include "tc_math.cuh"

namespace tc {

// In global memory (read through L1): every lane reads a different entry, which the constant
// cache would serialise.
__device__ const BinomTable c_binom_f = make_binom_table();

struct Brick {
    double x0b, y0b;        // brick centre
    double rbrick;          // sqrt(2) * h * 3.5
    double xlo, xhi, ylo, yhi;
    double h;
};

// MRAG block layout: bs x bs targets per block (the reference's build-time BLOCKSIZE, 32 by
// default), cut into 8 x 8 bricks, bps = bs / 8 per side; brick q of a block sits at column
// q % bps, row q / bps (rows of bricks, treecode-force.cpp:110-111), and target (ix, iy) of
// block b at ix + bs (iy + bs b).  The sides are powers of two, kept as their logarithms.
struct BlockLayout {
    int lbs, lbps;   // log2 of the targets and of the bricks per block side
};

__device__ __forceinline__ void brick_of(const BlockLayout &L, int brick, int &blk, int &bx,
                                         int &by) {
    blk = brick >> (2 * L.lbps);
    const int q = brick & ((1 << (2 * L.lbps)) - 1);
    bx = (q & ((1 << L.lbps) - 1)) * TILE;
    by = (q >> L.lbps) * TILE;
}

// Output index of target (bx + tx, by + ty) of block blk.
__device__ __forceinline__ size_t target_index(const BlockLayout &L, int blk, int bx, int by,
                                               int tx, int ty) {
    return ((size_t)blk << (2 * L.lbs)) + ((by + ty) << L.lbs) + bx + tx;
}

__device__ __forceinline__ Brick brick_geometry(double x0, double y0, double h, int bx, int by) {
    Brick b;
    b.h = h;
    b.x0b = __fma_rn((double)bx + 3.5, h, x0);
    b.y0b = __fma_rn((double)by + 3.5, h, y0);
    b.rbrick = __dmul_rn(4.949747468305833, h);
    b.xlo = __fma_rn((double)bx, h, x0);
    b.xhi = __fma_rn((double)(bx + TILE - 1), h, x0);
    b.ylo = __fma_rn((double)by, h, y0);
    b.yhi = __fma_rn((double)(by + TILE - 1), h, y0);
    return b;
}

enum { K_E2L = 0, K_E2P = 1, K_P2P = 2, K_DESCEND = 3, K_SKIP = 4 };

__device__ __forceinline__ int classify(const TNode &nd, const Brick &b, double inv_theta,
                                        double theta2) {
    const double dx = __dsub_rn(b.x0b, nd.xcom), dy = __dsub_rn(b.y0b, nd.ycom);
    const double dist = __dsqrt_rn(__fma_rn(dx, dx, __dmul_rn(dy, dy)));
    if (__dsub_rn(__ddiv_rn(dist, nd.r), 1.0) > inv_theta && b.rbrick <= nd.r) return K_E2L;
    const double xt = fmax(b.xlo, fmin(b.xhi, nd.xcom));
    const double yt = fmax(b.ylo, fmin(b.yhi, nd.ycom));
    const double ex = __dsub_rn(xt, nd.xcom), ey = __dsub_rn(yt, nd.ycom);
    const double r2 = __fma_rn(ex, ex, __dmul_rn(ey, ey));
    if (__dmul_rn(nd.r, nd.r) < __dmul_rn(theta2, r2)) return K_E2P;
    if (nd.child < 0) return nd.count > 0 ? K_P2P : K_SKIP;
    return K_DESCEND;
}

constexpr int TR_WARPS = 4;
constexpr int TR_STACK = 2048;
// A brick's evaluation is split into tasks of at most P2P_SEG near-field sources (task 0 also
// does the far field), so that the few bricks on a dense region do not serialise the kernel.
constexpr int P2P_SEG = 2048;
// Runs of blocks whose outputs are copied to the host while the next run is evaluated.
constexpr int FORCE_CHUNKS = 4;

// MODE 1: write the lists at the scanned offsets (CSR); MODE 2: count them and write each
// warp's entries into its own scratch region (ScratchLayout), recording where each brick's run
// starts, so that a copy into CSR order replaces a second walk.  A region that fills up sets
// meta[0] (the host then falls back to MODE 1); meta[1 + k] receives the longest run of kind k
// any warp wrote, for sizing the regions of the next build.
template <int MODE>
__global__ __launch_bounds__(TR_WARPS * 32) void k_force_lists(
    int nbricks, BlockLayout L, const double *__restrict__ x0s, const double *__restrict__ y0s,
    const double *__restrict__ hs, double theta, const TNode *__restrict__ tnode, int nnodes,
    int *__restrict__ counts, const int *__restrict__ offs, int *__restrict__ lists,
    int *__restrict__ scratch, ScratchLayout sl, int *__restrict__ sstart, int *meta,
    unsigned *err, unsigned long long *stats, int stack_cap) {
    constexpr bool FILL = MODE == 1;
    __shared__ int stack_all[TR_WARPS][TR_STACK];
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    int *stack = stack_all[warp];
    const double inv_theta = 1.0 / theta, theta2 = theta * theta;
    const unsigned lt = lanemask_lt();
    unsigned long long p2p_sources = 0;   // per lane: sources of the P2P leaves it listed
    const int wglob = blockIdx.x * TR_WARPS + warp;
    int cur[3] = {0, 0, 0};               // MODE 2: entries this warp has written, per kind
    bool full = false;

    for (int brick = blockIdx.x * TR_WARPS + warp; brick < nbricks;
         brick += gridDim.x * TR_WARPS) {
        int blk, bx, by;
        brick_of(L, brick, blk, bx, by);
        const Brick b = brick_geometry(x0s[blk], y0s[blk], hs[blk], bx, by);
        int o[3] = {0, 0, 0}, lim[3] = {0, 0, 0};
        if (FILL) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                o[k] = offs[k * nbricks + brick];
                lim[k] = offs[k * nbricks + brick + 1];
            }
        }
        int n[3] = {0, 0, 0};
        int bsrc = 0;   // per lane: sources of the P2P leaves it classified for this brick
        if (lane == 0) stack[0] = 0;
        int top = 1;
        __syncwarp();
        while (top > 0) {
            const int take = min(top, 32);
            top -= take;
            int node = -1, kind = K_SKIP, child = -1;
            if (lane < take) {
                node = stack[top + lane];
                if ((unsigned)node < (unsigned)nnodes) {
                    const TNode nd = tnode[node];
                    kind = classify(nd, b, inv_theta, theta2);
                    child = nd.child;
                    if (kind == K_P2P) bsrc += nd.count;
                    if (MODE != 0 && kind == K_P2P && stats) p2p_sources += (unsigned)nd.count;
                    if (kind == K_DESCEND && (child <= node || child + 4 > nnodes)) {
                        atomicOr(err, DEVERR_BOUNDS);
                        kind = K_SKIP;
                    }
                } else {
                    atomicOr(err, DEVERR_BOUNDS);
                }
            }
            __syncwarp();
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const unsigned bal = __ballot_sync(FULL_MASK, kind == k);
                if (FILL && kind == k) {
                    const int at = o[k] + n[k] + __popc(bal & lt);
                    if (at < lim[k]) lists[at] = node;
                    else atomicOr(err, DEVERR_BOUNDS);
                }
                if (MODE == 2 && kind == k) {
                    const int at = cur[k] + n[k] + __popc(bal & lt);
                    if (at < sl.cap[k]) scratch[sl.koff[k] + (size_t)wglob * sl.cap[k] + at] = node;
                    else full = true;
                }
                n[k] += __popc(bal);
            }
            const unsigned bd = __ballot_sync(FULL_MASK, kind == K_DESCEND);
            const int nd4 = 4 * __popc(bd);
            if (top + nd4 > stack_cap) {
                if (lane == 0) atomicOr(err, DEVERR_STACK);
                break;
            }
            if (kind == K_DESCEND) {
                const int pos = top + 4 * __popc(bd & lt);
#pragma unroll
                for (int c = 0; c < 4; ++c) stack[pos + c] = child + c;
            }
            top += nd4;
            __syncwarp();
        }
        if (!FILL) {
            const int total = __reduce_add_sync(FULL_MASK, bsrc);
            if (lane == 0) {
                counts[brick] = n[0];
                counts[nbricks + brick] = n[1];
                counts[2 * nbricks + brick] = n[2];
                // evaluation tasks: the brick's P2P sources in segments of at most P2P_SEG
                counts[3 * nbricks + brick] = max(1, (total + P2P_SEG - 1) / P2P_SEG);
                if (MODE == 2)
                    for (int k = 0; k < 3; ++k)
                        sstart[k * nbricks + brick] = sl.koff[k] + wglob * sl.cap[k] + cur[k];
            }
            if (MODE == 2)
                for (int k = 0; k < 3; ++k) cur[k] += n[k];
        }
        __syncwarp();
    }
    if (MODE == 2) {
        if (__any_sync(FULL_MASK, full) && lane == 0) atomicOr(&meta[0], 1);
        if (lane == 0)
            for (int k = 0; k < 3; ++k) atomicMax(&meta[1 + k], cur[k]);
    }
    if (MODE != 0 && stats) {
        for (int m = 16; m; m >>= 1) p2p_sources += __shfl_xor_sync(FULL_MASK, p2p_sources, m);
        if (lane == 0 && p2p_sources) atomicAdd(&stats[STAT_P2P_SOURCES], p2p_sources);
    }
}

// The lists in CSR order from the scratch runs of k_force_lists<2>: warp per brick.
__global__ __launch_bounds__(256) void k_force_lists_copy(int nbricks,
                                                          const int *__restrict__ counts,
                                                          const int *__restrict__ offs,
                                                          const int *__restrict__ sstart,
                                                          const int *__restrict__ scratch,
                                                          int *__restrict__ lists) {
    const int lane = lane_id();
    for (int brick = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; brick < nbricks;
         brick += (gridDim.x * blockDim.x) >> 5)
        for (int k = 0; k < 3; ++k) {
            const int n = counts[k * nbricks + brick];
            const int *src = scratch + sstart[k * nbricks + brick];
            int *dst = lists + offs[k * nbricks + brick];
            for (int i = lane; i < n; i += 32) dst[i] = src[i];
        }
}

// ------------------------------------------------------------------------------ evaluation
// The far field and the near field are two kernels, each with its own register budget: the
// far field keeps the FP64 E2L binomials in registers, the near field runs at a higher
// occupancy.
//  * k_force_far: persistent warps take bricks from an atomic counter; per brick the local
//    expansion from the E2L list (lane l owns coefficient l), L2P, and E2P over the E2P list,
//    2 targets per lane, written to the outputs at ix + 32*(iy + 32*ib)
//    (treecode-force.cpp:191-197).
//  * k_force_near: persistent warps take tasks from an atomic counter; a task is a segment of
//    at most P2P_SEG sources of a brick's P2P list, so that the few bricks on a dense region do
//    not serialise the kernel.  Source tiles are staged in shared memory, the next tile loaded
//    into registers meanwhile.  A brick with one task adds its near field to the output; the
//    tasks of a multi-task brick write partial sums that k_force_gather_parts adds to the
//    output in task order, so results are deterministic.
constexpr int EV_WARPS = 4;
constexpr int EV_CHUNK = 32;
constexpr int NEAR_MIN_BLOCKS = 8;   // near field: at most 64 registers per thread

template <int P>
struct FarShared {
    cplx coef[P];                 // E2L: a_k z^-(k+1); E2P: (k+1) a_k
    cplx local[P + 1];            // local expansion L_1..L_P
    float4 coef32[P];             // mixed E2P: scaled coefficient j as (re, re, im, im)
    float2 cf[P];                 // mixed E2L: D_k u^(k+1)
    float4 lf[P + 1];             // mixed L2P: l M_l as (re, re, im, im)
};

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// z^e for 0 <= e < 32 by square-and-multiply, FP32
__device__ __forceinline__ float2 cpowf_int(float2 z, int e) {
    float2 r = make_float2(1.f, 0.f), b = z;
#pragma unroll
    for (int bit = 0; bit < 5; ++bit) {
        if (e & (1 << bit)) r = cmulf(r, b);
        b = cmulf(b, b);
    }
    return r;
}

// Near-field source tile.  Plain form: the sources' x, y, v.  Mixed form: for each source k of
// the tile its offsets from the brick's 8 target columns (dx[c][k]) and 8 target rows
// (dy[r][k]) as floats, and its value; read four sources at a time (16-byte loads), rows padded
// to 36 words so that the 8 columns (4 rows) a warp reads at once fall in distinct banks.
constexpr int NEAR_ROW = EV_CHUNK + 4;
template <bool MIXED>
struct NearShared {
    double2 sxy[EV_CHUNK];
    double sv[EV_CHUNK];
};
template <>
struct __align__(16) NearShared<true> {
    float dx[TILE][NEAR_ROW];
    float dy[TILE][NEAR_ROW];
    float v[EV_CHUNK];
    float ch[TILE], cl[TILE];     // c h as float hi + lo, c = 0..7 (the task's brick)
};

__device__ __forceinline__ float rcp_approx_f32(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Compensated accumulation: (hi, lo) += x with an error-free two-sum (Knuth).
__device__ __forceinline__ void two_sum_acc(float &hi, float &lo, float x) {
    const float s = hi + x;
    const float bb = s - hi;
    const float err = (hi - (s - bb)) + (x - bb);
    hi = s;
    lo += err;
}

// A double split into two floats whose sum is within ~2^-48 relative of it.
__device__ __forceinline__ void split_f32(double v, float &hi, float &lo) {
    hi = (float)v;
    lo = (float)(v - (double)hi);
}

// MIXED = false: plain FP64.  MIXED = true: E2L, L2P and E2P in FP32 on power-of-two scaled
// quantities (scaled multipole coefficients, scaled local coefficients, offsets over the
// brick's scale), the two targets of a lane side by side in paired-FP32 (f32x2) registers,
// E2P's per-cell terms in compensated FP32 sums per target.
// LBS > 0: the block layout of side 2^LBS fixed at compile time (the default side 32 has its
// own instances: the layout arithmetic on kernel arguments measured 3% slower); LBS = 0: the
// layout L given at run time.
template <int P, bool MIXED, int LBS>
__global__ __launch_bounds__(EV_WARPS * 32, MIXED ? 5 : 4) void k_force_far(
    int nbricks, BlockLayout L_arg, const double *__restrict__ x0s, const double *__restrict__ y0s,
    const double *__restrict__ hs, const TNode *__restrict__ tnode,
    const double *__restrict__ mass, const double *__restrict__ exps,
    const int *__restrict__ offs, const int *__restrict__ lists, double *__restrict__ xout,
    double *__restrict__ yout, int brick_lo, int brick_hi, int *brick_ctr,
    const float2 *__restrict__ sexp, const float *__restrict__ sscale) {
    const BlockLayout L = LBS ? BlockLayout{LBS, LBS - 3} : L_arg;
    __shared__ FarShared<P> shared[EV_WARPS];
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    FarShared<P> &sh = shared[warp];
    const int tx = lane & 7, ty = lane >> 3;   // targets (tx, ty) and (tx, ty + 4)

    // signed binomials of lane l = lane + 1: (-1)^k C(l+k-1, k-1), k = 1..P, in registers
    // (in shared memory, for a higher occupancy, the kernel measured 18% slower); the mixed
    // form's FP32 E2L uses them divided by k (its coefficients carry a factor k, see E2L)
    using bsg_t = typename std::conditional<MIXED, float, double>::type;
    bsg_t bsg[P];
    {
        const int l = lane < P ? lane + 1 : 1;
#pragma unroll
        for (int k = 1; k <= P; ++k) {
            const double b = (k & 1 ? -1.0 : 1.0) * c_binom_f.c[l + k - 1][k - 1];
            bsg[k - 1] = (bsg_t)(MIXED ? b / k : b);
        }
    }

    for (;;) {
        int brick = 0;
        if (lane == 0) brick = brick_lo + atomicAdd(brick_ctr, 1);
        brick = __shfl_sync(FULL_MASK, brick, 0);
        if (brick < brick_lo || brick >= brick_hi) break;   // (a counter not reset: no access)
        int blk, bx, by;
        brick_of(L, brick, blk, bx, by);
        const double h = hs[blk];
        const Brick b = brick_geometry(x0s[blk], y0s[blk], h, bx, by);
        double ax0 = 0, ay0 = 0, ax1 = 0, ay1 = 0;

        // ---------------- E2L: local expansion about the brick centre (force-kernels.m4:102-155)
        if constexpr (MIXED) {
            // FP32 on power-of-two scaled quantities: R the cell's scale, rho >= r_brick the
            // brick's, u = R / z0, w = rho / z0, D_k = (k+1) a_k / R^(k+1) (sexp).  Scaled local
            // coefficients M_l = L_l rho^(l-1) = (w^l / rho) [-m/l + sum_k (-1)^k C(l+k-1, k-1)
            // (D_{k-1} / k) u^k]: an E2L cell has d > 3 r and r >= r_brick, so every term is
            // bounded by the cell's mass times ((r + rho) / d)^(l+k) < (2/3)^(l+k) (up to the
            // roundings of R and rho), nothing over- or underflows FP32, and the rounding errors
            // stay relative to the terms.  Lane l - 1 forms M_l; L2P uses l M_l.
            const int beg = offs[brick], end = offs[brick + 1];
            float2 Ml = make_float2(0.f, 0.f);
            const int l = lane + 1;
            const float minv = -1.f / (float)l;
            int erho = 0;
            frexp(b.rbrick, &erho);
            const double rho = ldexp(1.0, erho);   // 2^e > r_brick
            TNode nd_n = {};
            double m_n = 0;
            float sc_n = 1.f;
            float2 c_n = make_float2(0.f, 0.f);
            auto fetch = [&](int at) {
                const int node = lists[at];
                nd_n = tnode[node];
                m_n = mass[node];
                sc_n = sscale[node];
                if (lane < P) c_n = sexp[(size_t)node * P + lane];
            };
            if (beg < end) fetch(beg);
            for (int it = beg; it < end; ++it) {
                const TNode nd = nd_n;
                const float m = (float)m_n;
                const double R = sc_n;
                const float2 dk = c_n;
                if (it + 1 < end) fetch(it + 1);
                const double zx = nd.xcom - b.x0b, zy = nd.ycom - b.y0b;
                const double iz = rcp_nr(zx * zx + zy * zy);
                const float2 u = make_float2((float)(R * zx * iz), (float)(-R * zy * iz));
                const float2 w = make_float2((float)(rho * zx * iz), (float)(-rho * zy * iz));
                __syncwarp();
                if (lane < P) sh.cf[lane] = cmulf(dk, cpowf_int(u, l));   // D_{l-1} u^l
                __syncwarp();
                if (lane < P) {
                    float tr = l == 1 ? -m : m * minv, ti = 0.f;
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        const float2 ck = sh.cf[k];
                        tr = fmaf(bsg[k], ck.x, tr);
                        ti = fmaf(bsg[k], ck.y, ti);
                    }
                    const float2 t = cmulf(make_float2(tr, ti), cpowf_int(w, l));
                    Ml.x += t.x;
                    Ml.y += t.y;
                }
            }
            __syncwarp();
            if (lane < P)
                sh.lf[lane + 1] = make_float4(l * Ml.x, l * Ml.x, l * Ml.y, l * Ml.y);
            __syncwarp();
            // L2P (force-kernels.m4:157-191): sum_l l M_l (z / rho)^(l-1) / rho, the lane's two
            // targets side by side in f32x2 registers
            const float inv_rho = (float)(1.0 / rho);
            const float zxr = (float)((-3.5 * h + tx * h) / rho);
            const float2 zre = make_float2(zxr, zxr);
            const float2 zim = make_float2((float)((-3.5 * h + ty * h) / rho),
                                           (float)((-3.5 * h + (ty + 4) * h) / rho));
            const float2 nzim = make_float2(-zim.x, -zim.y);
            const float4 top = sh.lf[P];
            float2 are = make_float2(top.x, top.y), aim = make_float2(top.z, top.w);
#pragma unroll
            for (int q = P - 1; q >= 1; --q) {
                const float4 c = sh.lf[q];
                const float2 nre = __ffma2_rn(are, zre, __ffma2_rn(aim, nzim, make_float2(c.x, c.y)));
                aim = __ffma2_rn(are, zim, __ffma2_rn(aim, zre, make_float2(c.z, c.w)));
                are = nre;
            }
            ax0 += (double)(are.x * inv_rho);
            ay0 -= (double)(aim.x * inv_rho);
            ax1 += (double)(are.y * inv_rho);
            ay1 -= (double)(aim.y * inv_rho);
        } else {
            const int beg = offs[brick], end = offs[brick + 1];
            cplx Lc = {0.0, 0.0};
            const int l = lane + 1;
            const double minv = -1.0 / l;
            // the next cell is loaded while the current one is used
            TNode nd_n = {};
            double m_n = 0, ar_n = 0, ai_n = 0;
            auto fetch = [&](int at) {
                const int node = lists[at];
                nd_n = tnode[node];
                m_n = mass[node];
                if (lane < P) {
                    const double *ex = exps + (size_t)node * 2 * P;
                    ar_n = ex[lane];
                    ai_n = ex[P + lane];
                }
            };
            if (beg < end) fetch(beg);
            for (int it = beg; it < end; ++it) {
                const TNode nd = nd_n;
                const double m = m_n;
                const cplx a = {ar_n, ai_n};
                if (it + 1 < end) fetch(it + 1);
                const double zx = nd.xcom - b.x0b, zy = nd.ycom - b.y0b;
                const double r2z0 = zx * zx + zy * zy;
                const cplx zinv = {zx / r2z0, -zy / r2z0};
                cplx zl = {0.0, 0.0};
                if (lane < P) {
                    zl = cpow_int(zinv, l);        // z0^-l
                    sh.coef[lane] = cmul(a, zl);   // C_l = a_{l-1} z0^-l
                }
                __syncwarp();
                if (lane < P) {
                    double tr = l == 1 ? -m : m * minv, ti = 0.0;
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        const cplx ck = sh.coef[k];
                        tr = fma(bsg[k], ck.re, tr);
                        ti = fma(bsg[k], ck.im, ti);
                    }
                    Lc = cfma({tr, ti}, zl, Lc);
                }
                __syncwarp();
            }
            if (lane < P) sh.local[lane + 1] = Lc;
            __syncwarp();

            // L2P (force-kernels.m4:157-191): sum_l l L_l z^(l-1), z about the centre
            const double xr = -3.5 * h + tx * h;
            const double yr0 = -3.5 * h + ty * h, yr1 = -3.5 * h + (ty + 4) * h;
            cplx acc0 = {P * sh.local[P].re, P * sh.local[P].im}, acc1 = acc0;
            const cplx z0 = {xr, yr0}, z1 = {xr, yr1};
#pragma unroll
            for (int l = P - 1; l >= 1; --l) {
                const cplx cl = {l * sh.local[l].re, l * sh.local[l].im};
                acc0 = cfma(acc0, z0, cl);
                acc1 = cfma(acc1, z1, cl);
            }
            ax0 += acc0.re;
            ay0 -= acc0.im;
            ax1 += acc1.re;
            ay1 -= acc1.im;
        }

        // ---------------- E2P (force-kernels.m4:57-98): w = m/z - sum (j+1) a_j z^-(j+2)
        if (MIXED) {
            // FP32: u = 1/z, u' = R u with R the cell's power-of-two radius, scaled coefficients
            // D_j = (j+1) a_j / R^(j+1), w = u (m - u' Q(u')), Q(u') = sum_j D_j u'^j; the
            // Horner steps of the lane's two targets run side by side in f32x2 registers
            const int beg = offs[nbricks + brick], end = offs[nbricks + brick + 1];
            float hx0 = 0, lx0 = 0, hy0 = 0, ly0 = 0, hx1 = 0, lx1 = 0, hy1 = 0, ly1 = 0;
            TNode nd_n = {};
            double m_n = 0;
            float sc_n = 1.f;
            float2 c_n = make_float2(0.f, 0.f);
            auto fetch = [&](int at) {
                const int node = lists[at];
                nd_n = tnode[node];
                m_n = mass[node];
                sc_n = sscale[node];
                if (lane < P) c_n = sexp[(size_t)node * P + lane];
            };
            if (beg < end) fetch(beg);
            for (int it = beg; it < end; ++it) {
                const TNode nd = nd_n;
                const float m = (float)m_n, R = sc_n;
                __syncwarp();
                if (lane < P) sh.coef32[lane] = make_float4(c_n.x, c_n.x, c_n.y, c_n.y);
                __syncwarp();
                if (it + 1 < end) fetch(it + 1);
                const float rx = (float)((b.xlo - nd.xcom) + tx * h);
                const float ry0 = (float)((b.ylo - nd.ycom) + ty * h);
                const float ry1 = (float)((b.ylo - nd.ycom) + (ty + 4) * h);
                const float i0 = rcp_approx_f32(rx * rx + ry0 * ry0);
                const float i1 = rcp_approx_f32(rx * rx + ry1 * ry1);
                const float2 u0 = make_float2(rx * i0, -ry0 * i0), u1 = make_float2(rx * i1, -ry1 * i1);
                const float2 v0 = make_float2(R * u0.x, R * u0.y), v1 = make_float2(R * u1.x, R * u1.y);
                const float2 vre = make_float2(v0.x, v1.x), vim = make_float2(v0.y, v1.y);
                const float2 nvim = make_float2(-v0.y, -v1.y);
                const float4 top = sh.coef32[P - 1];
                float2 qre = make_float2(top.x, top.y), qim = make_float2(top.z, top.w);
#pragma unroll
                for (int j = P - 2; j >= 0; --j) {
                    const float4 d = sh.coef32[j];
                    const float2 nre = __ffma2_rn(qre, vre, __ffma2_rn(qim, nvim, make_float2(d.x, d.y)));
                    qim = __ffma2_rn(qre, vim, __ffma2_rn(qim, vre, make_float2(d.z, d.w)));
                    qre = nre;
                }
                const float2 q0 = make_float2(qre.x, qim.x), q1 = make_float2(qre.y, qim.y);
                const float t0x = m - (v0.x * q0.x - v0.y * q0.y), t0y = -(v0.x * q0.y + v0.y * q0.x);
                const float t1x = m - (v1.x * q1.x - v1.y * q1.y), t1y = -(v1.x * q1.y + v1.y * q1.x);
                two_sum_acc(hx0, lx0, u0.x * t0x - u0.y * t0y);
                two_sum_acc(hy0, ly0, -(u0.x * t0y + u0.y * t0x));
                two_sum_acc(hx1, lx1, u1.x * t1x - u1.y * t1y);
                two_sum_acc(hy1, ly1, -(u1.x * t1y + u1.y * t1x));
            }
            ax0 += (double)hx0 + (double)lx0;
            ay0 += (double)hy0 + (double)ly0;
            ax1 += (double)hx1 + (double)lx1;
            ay1 += (double)hy1 + (double)ly1;
        } else {
            const int beg = offs[nbricks + brick], end = offs[nbricks + brick + 1];
            // the next cell's record and coefficients are loaded while the current one is used
            TNode nd_n = {};
            double m_n = 0, cr_n = 0, ci_n = 0;
            auto fetch = [&](int at) {
                const int node = lists[at];
                nd_n = tnode[node];
                m_n = mass[node];
                if (lane < P) {
                    const double *ex = exps + (size_t)node * 2 * P;
                    cr_n = (lane + 1) * ex[lane];
                    ci_n = (lane + 1) * ex[P + lane];
                }
            };
            if (beg < end) fetch(beg);
            for (int it = beg; it < end; ++it) {
                const TNode nd = nd_n;
                const double m = m_n;
                __syncwarp();
                if (lane < P) sh.coef[lane] = {cr_n, ci_n};
                __syncwarp();
                if (it + 1 < end) fetch(it + 1);
                const double rx = (b.xlo - nd.xcom) + tx * h;
                const double ry0 = (b.ylo - nd.ycom) + ty * h;
                const double ry1 = (b.ylo - nd.ycom) + (ty + 4) * h;
                const double i0 = rcp_nr(rx * rx + ry0 * ry0);
                const double i1 = rcp_nr(rx * rx + ry1 * ry1);
                const cplx u0 = {rx * i0, -ry0 * i0}, u1 = {rx * i1, -ry1 * i1};
                cplx q0 = sh.coef[P - 1], q1 = q0;
#pragma unroll
                for (int j = P - 2; j >= 0; --j) {
                    const cplx d = sh.coef[j];
                    q0 = cfma(q0, u0, d);
                    q1 = cfma(q1, u1, d);
                }
                // w = u (m - u q)
                const cplx t0 = cmul(u0, q0), t1 = cmul(u1, q1);
                const cplx w0 = cmul(u0, {m - t0.re, -t0.im});
                const cplx w1 = cmul(u1, {m - t1.re, -t1.im});
                ax0 += w0.re;
                ay0 -= w0.im;
                ax1 += w1.re;
                ay1 -= w1.im;
            }
        }

        // the far field alone, in the output layout; k_add_far adds it to the near field
        const size_t o0 = target_index(L, blk, bx, by, tx, ty);
        const size_t o1 = o0 + ((size_t)4 << L.lbs);
        xout[o0] = ax0;
        yout[o0] = ay0;
        xout[o1] = ax1;
        yout[o1] = ay1;
        __syncwarp();
    }
}

// P2P (force-kernels.m4:15-55): sum v (xr, yr) / (xr^2 + yr^2 + eps) over the sources of a
// task's segment.  Both forms take one reciprocal per source for both of the lane's targets,
// 1/d0 = d1 / (d0 d1).
//  * MIXED = false: FP64, the reciprocal refined by two Newton steps (the squared separations
//    are at least eps and, for coordinates below ~1e70, their product stays far from the
//    double range's ends).
//  * MIXED = true: FP32 pairs on offsets from the brick corner (each source's offset to every
//    target column and row formed once per tile from float hi + lo parts, so the separation
//    keeps a few float ulps of itself), two sources per step in f32x2 registers, FP32 sums per
//    tile added into compensated per-target sums.
template <bool MIXED, int LBS>
__global__ __launch_bounds__(EV_WARPS * 32, NEAR_MIN_BLOCKS) void k_force_near(
    int nbricks, BlockLayout L_arg, const double *__restrict__ x0s, const double *__restrict__ y0s,
    const double *__restrict__ hs, const int2 *__restrict__ range, const double *__restrict__ xs,
    const double *__restrict__ ys, const double *__restrict__ vs, const int *__restrict__ offs,
    const int *__restrict__ lists, double *__restrict__ xout, double *__restrict__ yout,
    double *__restrict__ partial, int brick_lo, int brick_hi, int *task_ctr,
    const int *__restrict__ task_brick) {
    const BlockLayout L = LBS ? BlockLayout{LBS, LBS - 3} : L_arg;
    __shared__ NearShared<MIXED> shared[EV_WARPS];
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    NearShared<MIXED> &sh = shared[warp];
    const int tx = lane & 7, ty = lane >> 3;   // targets (tx, ty) and (tx, ty + 4)
    const double eps = 10 * DBL_EPSILON;

    // Tasks: brick b owns tasks [toff[b], toff[b+1]) (relative to toff[0]); task p covers
    // sources [p * P2P_SEG, (p + 1) * P2P_SEG) of the brick's P2P sequence.  This launch
    // evaluates the tasks of bricks [brick_lo, brick_hi).
    const int *toff = offs + 3 * nbricks;
    const int tbase = toff[0];
    const int task_lo = toff[brick_lo] - tbase, task_hi = toff[brick_hi] - tbase;
    for (;;) {
        int task = 0;
        if (lane == 0) task = task_lo + atomicAdd(task_ctr, 1);
        task = __shfl_sync(FULL_MASK, task, 0);
        if (task < task_lo || task >= task_hi) break;
        const int brick = task_brick[task];
        const int part = task - (toff[brick] - tbase);
        const int nparts = toff[brick + 1] - toff[brick];
        const int beg = offs[2 * nbricks + brick], end = offs[2 * nbricks + brick + 1];
        int blk, bx, by;
        brick_of(L, brick, blk, bx, by);
        const double h = hs[blk];
        const Brick b = brick_geometry(x0s[blk], y0s[blk], h, bx, by);
        double ax0 = 0, ay0 = 0, ax1 = 0, ay1 = 0;

        // Tiles of up to EV_CHUNK consecutive sources walk the listed leaves in order.
        int it = beg, s_next = 0, e_next = 0;
        auto take = [&]() { return range[lists[it++]]; };
        int skip = part * P2P_SEG, budget = P2P_SEG;
        while (it < end) {
            const int2 rg = take();
            const int cnt = rg.y - rg.x;
            if (skip < cnt) {
                s_next = rg.x + skip;
                e_next = rg.y;
                break;
            }
            skip -= cnt;
        }
        auto next_tile = [&](int &t0, int &tn) {
            while (s_next >= e_next && it < end) {
                const int2 rg = take();
                s_next = rg.x;
                e_next = rg.y;
            }
            t0 = s_next;
            tn = min(min(EV_CHUNK, e_next - s_next), budget);
            if (tn < 0) tn = 0;
            s_next += tn;
            budget -= tn;
        };
        int t0, tn;
        next_tile(t0, tn);
        double px = 0, py = 0, pv = 0;
        if (lane < tn) {
            px = xs[t0 + lane];
            py = ys[t0 + lane];
            pv = vs[t0 + lane];
        }
        if constexpr (MIXED) {
            const float epsf = (float)eps;
            const float2 eps2 = make_float2(epsf, epsf);
            float hx0 = 0, lx0 = 0, hy0 = 0, ly0 = 0, hx1 = 0, lx1 = 0, hy1 = 0, ly1 = 0;
            if (lane < TILE) split_f32(lane * h, sh.ch[lane], sh.cl[lane]);
            while (tn > 0) {
                const int cnt = tn;
                __syncwarp();
                {
                    // offsets of source `lane` from every target column / row: (c h - q) with
                    // q = source - corner, both as float hi + lo, two columns (rows) per f32x2
                    // instruction; slots past the tile get a zero value (their offsets, of an
                    // earlier source or of the origin, stay finite and their separations at
                    // least eps), so steps may take two sources at a time
                    float qxh, qxl, qyh, qyl;
                    split_f32(px - b.xlo, qxh, qxl);
                    split_f32(py - b.ylo, qyh, qyl);
                    const bool live = lane < cnt;
                    const float2 nqxh = make_float2(-qxh, -qxh), nqxl = make_float2(-qxl, -qxl);
                    const float2 nqyh = make_float2(-qyh, -qyh), nqyl = make_float2(-qyl, -qyl);
                    const float2 *ch2 = reinterpret_cast<const float2 *>(sh.ch);
                    const float2 *cl2 = reinterpret_cast<const float2 *>(sh.cl);
#pragma unroll
                    for (int c = 0; c < TILE; c += 2) {
                        const float2 ch = ch2[c >> 1], cl = cl2[c >> 1];
                        const float2 dx = __fadd2_rn(__fadd2_rn(ch, nqxh), __fadd2_rn(cl, nqxl));
                        const float2 dy = __fadd2_rn(__fadd2_rn(ch, nqyh), __fadd2_rn(cl, nqyl));
                        sh.dx[c][lane] = dx.x;
                        sh.dx[c + 1][lane] = dx.y;
                        sh.dy[c][lane] = dy.x;
                        sh.dy[c + 1][lane] = dy.y;
                    }
                    sh.v[lane] = live ? (float)pv : 0.f;
                }
                __syncwarp();
                next_tile(t0, tn);
                if (lane < tn) {
                    px = xs[t0 + lane];
                    py = ys[t0 + lane];
                    pv = vs[t0 + lane];
                }
                const float4 *dxr = reinterpret_cast<const float4 *>(sh.dx[tx]);
                const float4 *dyr0 = reinterpret_cast<const float4 *>(sh.dy[ty]);
                const float4 *dyr1 = reinterpret_cast<const float4 *>(sh.dy[ty + 4]);
                const float4 *vr4 = reinterpret_cast<const float4 *>(sh.v);
                float2 fx0 = make_float2(0.f, 0.f), fy0 = fx0, fx1 = fx0, fy1 = fx0;
                auto pairs = [&](float2 dx, float2 dy0, float2 dy1, float2 v) {
                    const float2 dx2e = __ffma2_rn(dx, dx, eps2);
                    const float2 d0 = __ffma2_rn(dy0, dy0, dx2e);
                    const float2 d1 = __ffma2_rn(dy1, dy1, dx2e);
                    const float2 p = __fmul2_rn(d0, d1);
                    const float2 r = make_float2(rcp_approx_f32(p.x), rcp_approx_f32(p.y));
                    const float2 vr = __fmul2_rn(v, r);
                    const float2 f0 = __fmul2_rn(vr, d1), f1 = __fmul2_rn(vr, d0);
                    fx0 = __ffma2_rn(dx, f0, fx0);
                    fy0 = __ffma2_rn(dy0, f0, fy0);
                    fx1 = __ffma2_rn(dx, f1, fx1);
                    fy1 = __ffma2_rn(dy1, f1, fy1);
                };
                const int nquad = (cnt + 3) >> 2;
#pragma unroll 2
                for (int k = 0; k < nquad; ++k) {
                    const float4 dx = dxr[k], dy0 = dyr0[k], dy1 = dyr1[k], v = vr4[k];
                    pairs(make_float2(dx.x, dx.y), make_float2(dy0.x, dy0.y),
                          make_float2(dy1.x, dy1.y), make_float2(v.x, v.y));
                    pairs(make_float2(dx.z, dx.w), make_float2(dy0.z, dy0.w),
                          make_float2(dy1.z, dy1.w), make_float2(v.z, v.w));
                }
                two_sum_acc(hx0, lx0, fx0.x + fx0.y);
                two_sum_acc(hy0, ly0, fy0.x + fy0.y);
                two_sum_acc(hx1, lx1, fx1.x + fx1.y);
                two_sum_acc(hy1, ly1, fy1.x + fy1.y);
            }
            ax0 = (double)hx0 + (double)lx0;
            ay0 = (double)hy0 + (double)ly0;
            ax1 = (double)hx1 + (double)lx1;
            ay1 = (double)hy1 + (double)ly1;
        } else {
            const double xt = b.xlo + tx * h;
            const double yt0 = b.ylo + ty * h, yt1 = b.ylo + (ty + 4) * h;
            while (tn > 0) {
                const int cnt = tn;
                __syncwarp();
                sh.sxy[lane] = make_double2(px, py);
                sh.sv[lane] = pv;
                __syncwarp();
                next_tile(t0, tn);
                if (lane < tn) {
                    px = xs[t0 + lane];
                    py = ys[t0 + lane];
                    pv = vs[t0 + lane];
                }
#pragma unroll 4
                for (int k = 0; k < cnt; ++k) {
                    const double2 sp = sh.sxy[k];
                    const double v = sh.sv[k];
                    const double xr = xt - sp.x;
                    const double xr2e = fma(xr, xr, eps);
                    const double yr0 = yt0 - sp.y, yr1 = yt1 - sp.y;
                    const double d0 = fma(yr0, yr0, xr2e), d1 = fma(yr1, yr1, xr2e);
                    const double vr = v * rcp_nr(d0 * d1);
                    const double f0 = vr * d1, f1 = vr * d0;
                    ax0 = fma(xr, f0, ax0);
                    ay0 = fma(yr0, f0, ay0);
                    ax1 = fma(xr, f1, ax1);
                    ay1 = fma(yr1, f1, ay1);
                }
            }
        }

        if (nparts == 1) {
            const size_t o0 = target_index(L, blk, bx, by, tx, ty);
            const size_t o1 = o0 + ((size_t)4 << L.lbs);
            xout[o0] = ax0;
            yout[o0] = ay0;
            xout[o1] = ax1;
            yout[o1] = ay1;
        } else {
            // partial result of this task; k_force_gather_parts adds the parts in order
            double *pp = partial + (size_t)task * 4 * 32;
            pp[lane] = ax0;
            pp[32 + lane] = ay0;
            pp[64 + lane] = ax1;
            pp[96 + lane] = ay1;
        }
        __syncwarp();
    }
}

// out += far over [begin, begin + count) of both output arrays (the near field plus the far
// field; the two kernels write separate buffers so that they need not wait for each other).
__global__ __launch_bounds__(256) void k_add_far(double *__restrict__ xout,
                                                 double *__restrict__ yout,
                                                 const double *__restrict__ xfar,
                                                 const double *__restrict__ yfar, size_t begin,
                                                 size_t count) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        xout[begin + i] += xfar[begin + i];
        yout[begin + i] += yfar[begin + i];
    }
}

// task -> brick map of the evaluation tasks
__global__ void k_task_map(int nbricks, const int *__restrict__ offs, int *__restrict__ task_brick) {
    const int *toff = offs + 3 * nbricks;
    const int tbase = toff[0];
    for (int brick = blockIdx.x * blockDim.x + threadIdx.x; brick < nbricks;
         brick += gridDim.x * blockDim.x)
        for (int t = toff[brick]; t < toff[brick + 1]; ++t) task_brick[t - tbase] = brick;
}

// Mixed form: multipole coefficients scaled by the cell's power-of-two radius R >= r,
// D_k = f_k a_k / R^(k+1) in FP32 (f_k = k + 1 for the force's derivative series, 1 for the
// potential), so that they stay O(mass) whatever the cell size; sscale = R.
template <int P, bool DERIV>
__global__ void k_scale_coeffs(int nnodes, const TNode *__restrict__ tnode,
                               const double *__restrict__ exps, float2 *__restrict__ sexp,
                               float *__restrict__ sscale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)nnodes * P;
         i += (long long)gridDim.x * blockDim.x) {
        const int node = (int)(i / P), k = (int)(i % P);
        const double r = tnode[node].r;
        int e = 0;
        if (r > 0 && r < 1e300) frexp(r, &e);   // r = f 2^e with f in [0.5, 1): 2^e >= r
        const double *ex = exps + (size_t)node * 2 * P;
        const double f = DERIV ? (double)(k + 1) : 1.0;
        sexp[i] = make_float2((float)(f * ldexp(ex[k], -e * (k + 1))),
                              (float)(f * ldexp(ex[P + k], -e * (k + 1))));
        if (k == 0) sscale[node] = (float)ldexp(1.0, e);
    }
}

// The near field of every multi-task brick: its parts added in task order (deterministic).
__global__ void k_force_gather_parts(int nbricks, int brick_lo, int brick_hi, BlockLayout L,
                                     const int *__restrict__ offs,
                                     const double *__restrict__ partial, double *__restrict__ xout,
                                     double *__restrict__ yout) {
    const int lane = lane_id();
    const int *toff = offs + 3 * nbricks;
    const int tbase = toff[0];
    for (int brick = brick_lo + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); brick < brick_hi;
         brick += (gridDim.x * blockDim.x) >> 5) {
        const int t0 = toff[brick] - tbase, np = toff[brick + 1] - toff[brick];
        if (np <= 1) continue;
        const int tx = lane & 7, ty = lane >> 3;
        int blk, bx, by;
        brick_of(L, brick, blk, bx, by);
        const size_t o0 = target_index(L, blk, bx, by, tx, ty);
        const size_t o1 = o0 + ((size_t)4 << L.lbs);
        // the parts in task order
        double ax0 = 0, ay0 = 0, ax1 = 0, ay1 = 0;
        for (int p = 0; p < np; ++p) {
            const double *pp = partial + (size_t)(t0 + p) * 4 * 32;
            ax0 += pp[lane];
            ay0 += pp[32 + lane];
            ax1 += pp[64 + lane];
            ay1 += pp[96 + lane];
        }
        xout[o0] = ax0;
        yout[o0] = ay0;
        xout[o1] = ax1;
        yout[o1] = ay1;
    }
}

static int sm_count() { return device_sm_count(); }

// The lists are counted, scanned and filled on the auxiliary stream; `between` (the expansion
// work, which the traversal does not read) runs on the main stream meanwhile, and the
// evaluation waits for both.
int force_mrag(Context &c, double theta, const double *x0s, const double *y0s, const double *hs,
               int nblocks, double *xout, double *yout, OverlapFn between, double *host_x,
               double *host_y) {
    BlockLayout L = {0, 0};
    while ((1 << L.lbs) < c.blocksize) ++L.lbs;   // 8, 16, 32 or 64 (tc_set_blocksize)
    L.lbps = L.lbs - 3;
    const int nbricks = nblocks << (2 * L.lbps);
    if (nbricks == 0) return TC_OK;
    int rc;
    // counts / offsets: E2L | E2P | P2P list lengths and evaluation tasks, nbricks each
    int *counts, *offs;
    if ((rc = ensure(c, S_FCOUNT, (size_t)4 * nbricks, &counts)) ||
        (rc = ensure(c, S_FOFF, (size_t)4 * nbricks + 1, &offs)))
        return rc;
    const TNode *tnode = slot_ptr<TNode>(c, S_TNODE);
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);
    const int trgrid = (int)std::min<long long>((nbricks + TR_WARPS - 1) / TR_WARPS,
                                                (long long)sm_count() * 16);
    // One walk counts the lists and writes them into per-warp scratch runs; after the scan a
    // copy puts them in CSR order.  If a run outgrew its region the second walk (MODE 1) writes
    // them instead, and the regions are sized up for the next solve.  The runs live in the
    // sort's record buffer when they fit in it, else in a block held only for the build.
    const int nwarps = trgrid * TR_WARPS;
    ScratchLayout sl;
    ListScratch ls;   // released (when transient) after the copy, in stream order
    int *sstart, *meta;
    {
        AuxScope on_aux(c);
        if ((rc = list_scratch(c, 3, nwarps, nbricks, sizeof(int), sl, ls)) ||
            (rc = ensure(c, S_LSTART, (size_t)3 * nbricks, &sstart)) ||
            (rc = ensure(c, S_LMETA, 4, &meta)))
            return rc;
    }
    unsigned long long *stats = slot_ptr<unsigned long long>(c, S_STATS);
    // traversal stack entries per warp: all of them, or fewer as a context's test setting
    const int stack_cap = c.stack_limit > 0 ? std::min(c.stack_limit, TR_STACK) : TR_STACK;
    TC_CUDA_TRY(cudaEventRecord(c.ev_fork, c.stream));
    {
        AuxScope on_aux(c);
        TC_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.ev_fork, 0));
        TC_CUDA_TRY(cudaMemsetAsync(meta, 0, sizeof(int) * 4, c.stream));
        k_force_lists<2><<<trgrid, TR_WARPS * 32, 0, c.stream>>>(
            nbricks, L, x0s, y0s, hs, theta, tnode, c.nnodes, counts, nullptr, nullptr,
            static_cast<int *>(ls.p), sl, sstart, meta, err, stats, stack_cap);
        TC_KERNEL_CHECK();
        if ((rc = exclusive_scan(c, counts, offs, 4 * nbricks))) return rc;
        for (int k = 0; k < 4; ++k)
            TC_CUDA_TRY(cudaMemcpyAsync(c.h_pinned + 32 + k, offs + (k + 1) * nbricks, sizeof(int),
                                        cudaMemcpyDeviceToHost, c.stream));
        TC_CUDA_TRY(cudaMemcpyAsync(c.h_pinned + 36, meta, sizeof(int) * 4,
                                    cudaMemcpyDeviceToHost, c.stream));
        TC_CUDA_TRY(cudaEventRecord(c.ev_totals, c.stream));
    }
    if (between && (rc = between(c))) {
        cudaStreamSynchronize(c.aux);   // leave nothing of this solve in flight
        return rc;
    }
    TC_CUDA_TRY(wait_event(c, c.ev_totals));
    int tot[4];
    for (int k = 0; k < 4; ++k) tot[k] = (int)c.h_pinned[32 + k];
    const bool overflow = c.h_pinned[36] != 0;
    c.list_walks = overflow ? 2 : 1;
    scratch_learn(c, 3, nwarps, nbricks, c.h_pinned + 37);   // for the next solve
    const int ntasks = tot[3] - tot[2];
    c.counts.n_e2l = tot[0];
    c.counts.n_e2p = tot[1] - tot[0];
    c.counts.n_p2p = tot[2] - tot[1];
    c.counts.e2l_pairs = c.counts.n_e2l;
    c.counts.e2p_pairs = c.counts.n_e2p * TILE * TILE;
    c.counts.l2p_targets = (long long)nbricks * TILE * TILE;
    int *lists;
    {
        AuxScope on_aux(c);
        if ((rc = ensure(c, S_E2L, (size_t)tot[2] + 1, &lists))) return rc;
        if (!overflow) {
            k_force_lists_copy<<<(int)std::min<long long>((nbricks + 7) / 8,
                                                          (long long)sm_count() * 16),
                                 256, 0, c.stream>>>(nbricks, counts, offs, sstart,
                                                     static_cast<const int *>(ls.p), lists);
        } else {
            k_force_lists<1><<<trgrid, TR_WARPS * 32, 0, c.stream>>>(
                nbricks, L, x0s, y0s, hs, theta, tnode, c.nnodes, nullptr, offs, lists, nullptr,
                sl, nullptr, nullptr, err, nullptr, stack_cap);
        }
        TC_KERNEL_CHECK();
        TC_CUDA_TRY(cudaEventRecord(c.ev_join, c.stream));
    }
    // The near field reads the sources and the P2P lists only, not the expansions: it runs on
    // the auxiliary stream as soon as the lists are in place, while the upward pass forms the
    // expansions and the far field is evaluated on the main stream.  The near field writes the
    // outputs, the far field buffers of its own, and k_add_far adds the two once both are done.
    int *brick_ctr, *task_brick;
    // (measurement mode: the near field waits for the upward pass, the far field for it)
    if (c.serial_eval) TC_CUDA_TRY(cudaEventRecord(c.ev_serial, c.stream));
    {
        AuxScope on_aux(c);
        if (c.serial_eval) TC_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.ev_serial, 0));
        // everything the near field uses is allocated and written on this stream (the far
        // field's work counters are the main stream's own, S_FAR_CTR)
        double *partial;
        if ((rc = ensure(c, S_BRICK_CTR, 1, &brick_ctr)) ||
            (rc = ensure(c, S_FPART, (size_t)ntasks * 4 * 32, &partial)) ||
            (rc = ensure(c, S_TASKMAP, (size_t)ntasks, &task_brick)))
            return rc;
        TC_CUDA_TRY(cudaMemsetAsync(brick_ctr, 0, sizeof(int), c.stream));
        k_task_map<<<(int)std::min<long long>((nbricks + 255) / 256, (long long)sm_count() * 8),
                     256, 0, c.stream>>>(nbricks, offs, task_brick);
        TC_KERNEL_CHECK();
        const bool mixed = c.precision == 1;
        constexpr int LBS32 = 5;   // the default block side, 32
        const bool fixed = L.lbs == LBS32;
        auto near = mixed ? (fixed ? k_force_near<true, LBS32> : k_force_near<true, 0>)
                          : (fixed ? k_force_near<false, LBS32> : k_force_near<false, 0>);
        const int occ_near = mixed ? blocks_per_sm<k_force_near<true, LBS32>>(EV_WARPS * 32, 0)
                                   : blocks_per_sm<k_force_near<false, LBS32>>(EV_WARPS * 32, 0);
        const int neargrid = (int)std::min<long long>((ntasks + EV_WARPS - 1) / EV_WARPS,
                                                      (long long)sm_count() * occ_near);
        phase_mark(c, 9);
        near<<<neargrid, EV_WARPS * 32, 0, c.stream>>>(
            nbricks, L, x0s, y0s, hs, slot_ptr<int2>(c, S_RANGE), slot_ptr<double>(c, S_XS),
            slot_ptr<double>(c, S_YS), slot_ptr<double>(c, S_VS), offs, lists, xout, yout,
            partial, 0, nbricks, brick_ctr, task_brick);
        TC_KERNEL_CHECK();
        if (ntasks > nbricks) {
            k_force_gather_parts<<<(int)std::min<long long>((nbricks + 7) / 8,
                                                            (long long)sm_count() * 16),
                                   256, 0, c.stream>>>(nbricks, 0, nbricks, L, offs, partial, xout,
                                                       yout);
            TC_KERNEL_CHECK();
        }
        phase_mark(c, 10);
        c.near_marked = c.timing;
        TC_CUDA_TRY(cudaEventRecord(c.ev_near, c.stream));
    }
    TC_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.ev_join, 0));
    phase_mark(c, 4);
    // the evaluation for the tree's expansion order
    rc = dispatch_order(c.order, [&](auto order) -> int {
        constexpr int P = decltype(order)::value;
        int rc2;
        const bool mixed = c.precision == 1;
        float2 *sexp = nullptr;
        float *sscale = nullptr;
        if (mixed) {
            if ((rc2 = ensure(c, S_SEXP, (size_t)c.nnodes * P, &sexp)) ||
                (rc2 = ensure(c, S_SSCALE, (size_t)c.nnodes, &sscale)))
                return rc2;
            const long long items = (long long)c.nnodes * P;
            k_scale_coeffs<P, true>
                <<<(int)std::min<long long>((items + 255) / 256, (long long)sm_count() * 8), 256, 0,
                   c.stream>>>(c.nnodes, tnode, slot_ptr<double>(c, S_EXPS), sexp, sscale);
            TC_KERNEL_CHECK();
        }
        constexpr int LBS32 = 5;   // the default block side, 32
        const bool fixed = L.lbs == LBS32;
        auto far = mixed ? (fixed ? k_force_far<P, true, LBS32> : k_force_far<P, true, 0>)
                         : (fixed ? k_force_far<P, false, LBS32> : k_force_far<P, false, 0>);
        const int occ_far = mixed ? blocks_per_sm<k_force_far<P, true, LBS32>>(EV_WARPS * 32, 0)
                                  : blocks_per_sm<k_force_far<P, false, LBS32>>(EV_WARPS * 32, 0);
        const int fargrid = (int)std::min<long long>((nbricks + EV_WARPS - 1) / EV_WARPS,
                                                     (long long)sm_count() * occ_far);
        // With host outputs of 2^21 targets or more (a copy of >= 32 MB, ~0.6 ms over PCIe) the
        // blocks are evaluated in FORCE_CHUNKS runs, each copied to the host on the auxiliary
        // stream while the next one is evaluated; below that the runs' tails cost more than
        // the overlap gains (measured: 16M sheet e2e 11.07 -> 10.67 ms, 1M vortex 2.01 ->
        // 2.27 ms if split).
        const size_t per_block = (size_t)1 << (2 * L.lbs);
        const size_t nt_all = (size_t)nblocks * per_block;
        double *xfar, *yfar;
        int *far_ctr;
        if ((rc2 = ensure(c, S_FARX, nt_all, &xfar)) || (rc2 = ensure(c, S_FARY, nt_all, &yfar)) ||
            (rc2 = ensure(c, S_FAR_CTR, FORCE_CHUNKS, &far_ctr)))
            return rc2;
        TC_CUDA_TRY(cudaMemsetAsync(far_ctr, 0, FORCE_CHUNKS * sizeof(int), c.stream));
        const int nchunks =
            host_x && (size_t)nblocks * per_block >= ((size_t)1 << 21) && nblocks >= FORCE_CHUNKS
                ? FORCE_CHUNKS
                : 1;
        if (c.serial_eval) TC_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.ev_near, 0));
        phase_mark(c, 6);
        for (int k = 0; k < nchunks; ++k) {
            const int blk0 = (int)((long long)nblocks * k / nchunks);
            const int blk1 = (int)((long long)nblocks * (k + 1) / nchunks);
            const int b0 = blk0 << (2 * L.lbps), b1 = blk1 << (2 * L.lbps);
            far<<<fargrid, EV_WARPS * 32, 0, c.stream>>>(
                nbricks, L, x0s, y0s, hs, tnode, slot_ptr<double>(c, S_MASS),
                slot_ptr<double>(c, S_EXPS), offs, lists, xfar, yfar, b0, b1, far_ctr + k, sexp,
                sscale);
            TC_KERNEL_CHECK();
            if (k == nchunks - 1) phase_mark(c, 7);
            const size_t o = blk0 * per_block, cnt = (size_t)(blk1 - blk0) * per_block;
            if (k == 0) TC_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.ev_near, 0));
            k_add_far<<<(int)std::min<long long>((long long)(cnt + 255) / 256,
                                                 (long long)sm_count() * 8),
                        256, 0, c.stream>>>(xout, yout, xfar, yfar, o, cnt);
            TC_KERNEL_CHECK();
            if (nchunks > 1) {
                TC_CUDA_TRY(cudaEventRecord(c.ev_chunk[k], c.stream));
                TC_CUDA_TRY(cudaStreamWaitEvent(c.aux, c.ev_chunk[k], 0));
                TC_CUDA_TRY(cudaMemcpyAsync(host_x + o, xout + o, sizeof(double) * cnt,
                                            cudaMemcpyDeviceToHost, c.aux));
                TC_CUDA_TRY(cudaMemcpyAsync(host_y + o, yout + o, sizeof(double) * cnt,
                                            cudaMemcpyDeviceToHost, c.aux));
            }
        }
        c.host_copied = nchunks > 1;
        return TC_OK;
    });
    if (rc) return rc;
    return TC_OK;
}

void kernels_force(KernelList &v) {
    v.insert(v.end(), {(const void *)k_force_lists<1>, (const void *)k_force_lists<2>,
                       (const void *)k_force_lists_copy, (const void *)k_task_map,
                       (const void *)k_add_far,
                       (const void *)k_force_gather_parts, (const void *)k_force_near<true, 5>,
                       (const void *)k_force_near<true, 0>, (const void *)k_force_near<false, 5>,
                       (const void *)k_force_near<false, 0>});
#define TC_FORCE_KERNELS(P)                                                                      \
    v.insert(v.end(), {(const void *)k_force_far<P, true, 5>, (const void *)k_force_far<P, true, 0>, \
                       (const void *)k_force_far<P, false, 5>,                                   \
                       (const void *)k_force_far<P, false, 0>, (const void *)k_scale_coeffs<P, true>});
    TC_FOR_EACH_ORDER(TC_FORCE_KERNELS)
#undef TC_FORCE_KERNELS
}

}  // namespace tc
