// potential.cu -- treecode_potential on the GPU.
//
// Restates drivers/treecode-potential.cpp:25-87 (per-target traversal) and
// kernels/potential-kernels.m4 (P2P, E2P).  The opening test is per target
// (r^2 < theta^2 |t - com|^2, treecode-potential.cpp:48-50), so the warp-cooperative traversal
// keeps, for every stack entry, the mask of lanes (targets) that still need the node:
//   far  = lanes in the mask that accept the node            -> E2P entry (node, far)
//   rest = mask & ~far; leaf -> P2P entry (node, rest); inner -> push children with `rest`.
// Each target therefore sees exactly the nodes the reference's own DFS would give it.
// Targets are first sorted by Morton key (in the sources' frame) so that the 32 targets of a
// warp are neighbours and the masks are mostly full.
//
// Lists are (node, lane mask) pairs in CSR form per group of 32 targets, built by a counting
// walk, a scan, and a filling walk.
#include <cfloat>

#include "tc_internal.h"
#include "tc_math.cuh"

namespace tc {

constexpr int PT_WARPS = 4;
// A group's evaluation is split into tasks of at most PT_SEG near-field sources (task 0 also
// does the far field), so that groups inside dense clusters do not serialise the kernel.
constexpr int PT_SEG = 4096;

// Lists of one group of 32 targets.  The warp pops up to 32 stack entries (node, target mask)
// at a time, one per lane, so the latency of the node reads is shared by a whole batch.  A lane
// decides its node for the entry's targets with the group's bounding box first: when every
// point of the box is clearly far (or clearly near) -- with a relative margin of 1e-12, far
// above the rounding of the per-target test -- the whole mask follows; otherwise the exact
// per-target test (r^2 < theta^2 |t - com|^2, treecode-potential.cpp:48-50) runs for each
// target of the mask.  Far targets give an E2P entry (node, far); the rest give a P2P entry for
// a leaf or push the node's four children with the rest.  Every target thus gets exactly the
// nodes its own depth-first traversal in the reference would give it.  Entries are written in
// the (deterministic) processing order; the count pass and the fill pass take the same steps.
// Stack entries per warp.  A batch of nb entries pushes at most 4 nb, so batches are taken only
// while top <= PL_STACK - 160; above that the walk pops one entry at a time (depth first), which
// grows the stack by at most 3 per level, 45 in all, before it shrinks again.  The stack thus
// never holds more than PL_STACK - 160 + 96 + 45 entries.
constexpr int PL_STACK = 512;

// MODE 1: write the lists at the scanned offsets (CSR); MODE 2: count them and write each
// warp's entries into its own scratch region (ScratchLayout), recording where each group's run
// starts, so that a copy into CSR order replaces a second walk.  A region that fills up sets
// meta[0] (the host then falls back to MODE 1); meta[1 + k] receives the longest run of kind
// k any warp wrote.  The work counters are added by the walk that runs last over every group
// (MODE 2, or MODE 1 when it runs).
template <int MODE>
__global__ __launch_bounds__(PT_WARPS * 32) void k_potential_lists(
    int ngroups, int m, const double *__restrict__ xt, const double *__restrict__ yt,
    const int *__restrict__ tperm, double theta, const TNode *__restrict__ tnode, int nnodes,
    int *__restrict__ counts, const int *__restrict__ offs, int2 *__restrict__ lists,
    int2 *__restrict__ scratch, ScratchLayout sl, int *__restrict__ sstart, int *meta,
    unsigned *err, unsigned long long *stats) {
    constexpr bool FILL = MODE == 1;
    const int wglob = blockIdx.x * PT_WARPS + (threadIdx.x >> 5);
    int cur[2] = {0, 0};   // MODE 2: entries this warp has written, per kind
    bool full = false;
    __shared__ int2 stack_all[PT_WARPS][PL_STACK];
    __shared__ double2 targ_all[PT_WARPS][32];
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    int2 *stack = stack_all[warp];
    double2 *targ = targ_all[warp];
    const unsigned lt = (1u << lane) - 1u;
    const double theta2 = theta * theta;
    unsigned long long e2p_pairs = 0, p2p_pairs = 0;   // warp-uniform work counters

    for (int g = blockIdx.x * PT_WARPS + warp; g < ngroups; g += gridDim.x * PT_WARPS) {
        const int t = g * 32 + lane;
        const bool valid = t < m;
        double x = 0, y = 0;
        if (valid) {
            const int j = tperm[t];
            x = xt[j];
            y = yt[j];
        }
        const unsigned vmask = __ballot_sync(FULL_MASK, valid);
        // bounding box of the group's targets
        double bxlo = valid ? x : 1e300, bxhi = valid ? x : -1e300;
        double bylo = valid ? y : 1e300, byhi = valid ? y : -1e300;
        for (int o = 16; o; o >>= 1) {
            bxlo = fmin(bxlo, __shfl_xor_sync(FULL_MASK, bxlo, o));
            bxhi = fmax(bxhi, __shfl_xor_sync(FULL_MASK, bxhi, o));
            bylo = fmin(bylo, __shfl_xor_sync(FULL_MASK, bylo, o));
            byhi = fmax(byhi, __shfl_xor_sync(FULL_MASK, byhi, o));
        }
        int o0 = 0, o1 = 0, l0 = 0, l1 = 0;
        if (FILL) {
            o0 = offs[g];
            l0 = offs[g + 1];
            o1 = offs[ngroups + g];
            l1 = offs[ngroups + g + 1];
        }
        __syncwarp();
        targ[lane] = make_double2(x, y);
        if (lane == 0) stack[0] = make_int2(0, (int)vmask);
        __syncwarp();
        int n0 = 0, n1 = 0, gsrc = 0, top = 1;
        bool overflow = false;
        while (top > 0 && !overflow) {
            const int nb = top > PL_STACK - 160 ? 1 : min(32, top), base = top - nb;
            const bool act = lane < nb;
            int2 ent = make_int2(0, 0);
            if (act) ent = stack[base + lane];
            __syncwarp();
            top = base;
            const unsigned mask = (unsigned)ent.y;
            bool ok = act && mask != 0;
            if (act && (unsigned)ent.x >= (unsigned)nnodes) {
                atomicOr(err, DEVERR_BOUNDS);
                ok = false;
            }
            TNode nd = {};
            if (ok) nd = tnode[ent.x];
            unsigned far = 0;
            if (ok) {
                const double rr = __dmul_rn(nd.r, nd.r);
                const double ex = fmax(fmax(bxlo - nd.xcom, nd.xcom - bxhi), 0.0);
                const double ey = fmax(fmax(bylo - nd.ycom, nd.ycom - byhi), 0.0);
                const double fx = fmax(nd.xcom - bxlo, bxhi - nd.xcom);
                const double fy = fmax(nd.ycom - bylo, byhi - nd.ycom);
                const double dmin2 = ex * ex + ey * ey, dmax2 = fx * fx + fy * fy;
                if (rr < theta2 * dmin2 * (1.0 - 1e-12)) {
                    far = mask;                         // every target of the box is far
                } else if (rr >= theta2 * dmax2 * (1.0 + 1e-12)) {
                    far = 0;                            // every target of the box is near
                } else {
                    for (unsigned mm = mask; mm; mm &= mm - 1) {
                        const int tl = __ffs(mm) - 1;
                        const double2 tp = targ[tl];
                        // r2 without contraction, as the compiled reference
                        const double dx = __dsub_rn(tp.x, nd.xcom), dy = __dsub_rn(tp.y, nd.ycom);
                        const double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
                        if (rr < __dmul_rn(theta2, r2)) far |= 1u << tl;
                    }
                }
            }
            const unsigned rest = mask & ~far;
            const bool leaf = nd.child < 0;
            const bool f_far = ok && far != 0;
            const bool f_near = ok && rest != 0 && leaf && nd.count > 0;
            bool f_push = ok && rest != 0 && !leaf;
            if (f_push && (nd.child <= ent.x || nd.child + 4 > nnodes)) {
                atomicOr(err, DEVERR_BOUNDS);
                f_push = false;
            }
            const unsigned bf = __ballot_sync(FULL_MASK, f_far);
            const unsigned bn = __ballot_sync(FULL_MASK, f_near);
            const unsigned bp = __ballot_sync(FULL_MASK, f_push);
            if (FILL) {
                if (f_far) {
                    const int at = o0 + n0 + __popc(bf & lt);
                    if (at < l0) lists[at] = make_int2(ent.x, (int)far);
                    else atomicOr(err, DEVERR_BOUNDS);
                }
                if (f_near) {
                    const int at = o1 + n1 + __popc(bn & lt);
                    if (at < l1) lists[at] = make_int2(ent.x, (int)rest);
                    else atomicOr(err, DEVERR_BOUNDS);
                }
            }
            if (MODE == 2) {
                if (f_far) {
                    const int at = cur[0] + n0 + __popc(bf & lt);
                    if (at < sl.cap[0])
                        scratch[sl.koff[0] + (size_t)wglob * sl.cap[0] + at] =
                            make_int2(ent.x, (int)far);
                    else full = true;
                }
                if (f_near) {
                    const int at = cur[1] + n1 + __popc(bn & lt);
                    if (at < sl.cap[1])
                        scratch[sl.koff[1] + (size_t)wglob * sl.cap[1] + at] =
                            make_int2(ent.x, (int)rest);
                    else full = true;
                }
            }
            n0 += __popc(bf);
            n1 += __popc(bn);
            e2p_pairs += (unsigned)__reduce_add_sync(FULL_MASK, f_far ? __popc(far) : 0);
            const unsigned cnt = f_near ? (unsigned)nd.count : 0u;
            gsrc += (int)__reduce_add_sync(FULL_MASK, cnt);
            p2p_pairs += __reduce_add_sync(FULL_MASK, f_near ? (unsigned)__popc(rest) * cnt : 0u);
            const int npush = 4 * __popc(bp);
            if (top + npush > PL_STACK) {
                if (lane == 0) atomicOr(err, DEVERR_STACK);
                overflow = true;
            } else {
                if (f_push) {
                    const int at = top + 4 * __popc(bp & lt);
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        stack[at + c] = make_int2(nd.child + 3 - c, (int)rest);
                }
                top += npush;
            }
            __syncwarp();
        }
        if (!FILL && lane == 0) {
            counts[g] = n0;
            counts[ngroups + g] = n1;
            // evaluation tasks: the group's near-field sources in segments of at most PT_SEG
            counts[2 * ngroups + g] = max(1, (gsrc + PT_SEG - 1) / PT_SEG);
            if (MODE == 2) {
                sstart[g] = sl.koff[0] + wglob * sl.cap[0] + cur[0];
                sstart[ngroups + g] = sl.koff[1] + wglob * sl.cap[1] + cur[1];
            }
        }
        if (MODE == 2) {
            cur[0] += n0;
            cur[1] += n1;
        }
        __syncwarp();
    }
    if (MODE == 2) {
        if (__any_sync(FULL_MASK, full) && lane == 0) atomicOr(&meta[0], 1);
        if (lane == 0) {
            atomicMax(&meta[1], cur[0]);
            atomicMax(&meta[2], cur[1]);
        }
    }
    if (stats && lane == 0) {
        if (e2p_pairs) atomicAdd(&stats[STAT_E2P_PAIRS], e2p_pairs);
        if (p2p_pairs) atomicAdd(&stats[STAT_P2P_PAIRS], p2p_pairs);
    }
}

// The lists in CSR order from the scratch runs of k_potential_lists<2>: warp per group.
__global__ __launch_bounds__(256) void k_potential_lists_copy(int ngroups,
                                                              const int *__restrict__ counts,
                                                              const int *__restrict__ offs,
                                                              const int *__restrict__ sstart,
                                                              const int2 *__restrict__ scratch,
                                                              int2 *__restrict__ lists) {
    const int lane = lane_id();
    for (int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ngroups;
         g += (gridDim.x * blockDim.x) >> 5)
        for (int k = 0; k < 2; ++k) {
            const int n = counts[k * ngroups + g];
            const int2 *src = scratch + sstart[k * ngroups + g];
            int2 *dst = lists + offs[k * ngroups + g];
            for (int i = lane; i < n; i += 32) dst[i] = src[i];
        }
}

constexpr int PE_WARPS = 4;
constexpr int PE_CHUNK = 32;

__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void two_sum_add(float &hi, float &lo, float x) {
    const float s = hi + x;
    const float bb = s - hi;
    lo += (hi - (s - bb)) + (x - bb);
    hi = s;
}

__device__ __forceinline__ void split2(double v, float &hi, float &lo) {
    hi = (float)v;
    lo = (float)(v - (double)hi);
}

// Tasks: group g owns tasks [toff[g], toff[g+1]); task 0 evaluates the far field and the first
// PT_SEG near-field sources of the group, task p > 0 the p-th segment.
// MIXED = false: FP64 throughout (log of FP64).  MIXED = true: the series of E2P and the P2P
// logs in FP32 (offsets from the group's first target split hi + lo, lg2.approx, compensated
// sums); the monopole term m log|z| of E2P stays FP64.
template <int P, bool MIXED>
__global__ __launch_bounds__(PE_WARPS * 32) void k_potential_eval(
    int ngroups, int m, const double *__restrict__ xt, const double *__restrict__ yt,
    const int *__restrict__ tperm, const TNode *__restrict__ tnode,
    const double *__restrict__ mass, const double *__restrict__ exps,
    const int2 *__restrict__ range, const double *__restrict__ xs,
    const double *__restrict__ ys, const double *__restrict__ vs,
    const int *__restrict__ offs, const int2 *__restrict__ lists, double *__restrict__ out,
    double *__restrict__ partial, int *task_ctr, const int *__restrict__ task_group,
    const float2 *__restrict__ sexp, const float *__restrict__ sscale) {
    __shared__ cplx s_coef[PE_WARPS][P];
    // mixed E2P coefficients in pairs (D_2j.re, D_2j+1.re, D_2j.im, D_2j+1.im): the even and
    // the odd series run side by side in f32x2 lanes
    __shared__ float4 s_coef32[PE_WARPS][P / 2];
    __shared__ double2 s_xy[PE_WARPS][PE_CHUNK];
    __shared__ double s_v[PE_WARPS][PE_CHUNK];
    // mixed form: the tile as negated float offsets (hi + lo) from the group's reference point,
    // two sources per entry for paired-FP32 (f32x2) arithmetic: (-x hi, -x hi', -x lo, -x lo'),
    // the same for y, and (v, v')
    __shared__ float4 s_nx[PE_WARPS][PE_CHUNK / 2];
    __shared__ float4 s_ny[PE_WARPS][PE_CHUNK / 2];
    __shared__ float2 s_v2[PE_WARPS][PE_CHUNK / 2];
    __shared__ double s_part[PE_WARPS][32];        // P2P lane partials of a sparse mask
    __shared__ double s_neg_log_c[LOG_NTAB];       // log_pos's table
    load_log_table(s_neg_log_c);
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    const double eps = 10 * DBL_EPSILON;
    const int *toff = offs + 2 * ngroups;
    const int tbase = toff[0];
    const int ntasks = toff[ngroups] - tbase;

    for (;;) {
        int task = 0;
        if (lane == 0) task = atomicAdd(task_ctr, 1);
        task = __shfl_sync(FULL_MASK, task, 0);
        if (task >= ntasks) break;
        const int g = task_group[task];
        const int part = task - (toff[g] - tbase);
        const int nparts = toff[g + 1] - toff[g];
        const int t = g * 32 + lane;
        const bool valid = t < m;
        int j = 0;
        double x = 0, y = 0;
        if (valid) {
            j = tperm[t];
            x = xt[j];
            y = yt[j];
        }
        // reference point of the mixed form's offsets: the group's first target
        const double xref = __shfl_sync(FULL_MASK, x, 0), yref = __shfl_sync(FULL_MASK, y, 0);
        double far = 0, near = 0;

        // E2P (potential-kernels.m4:59-89): m log(r2)/2 + Re sum_{j=1..p} a_{j-1} z^-j.  The next
        // entry's cell record and coefficients are loaded while the current one is evaluated.
        if (part == 0) {
            const int b0 = offs[g], e0 = offs[g + 1];
            float sh = 0, sl = 0;
            int2 ent_n = make_int2(0, 0);
            TNode nd_n = {};
            double m_n = 0, cr_n = 0, ci_n = 0;
            float R_n = 1.f;
            float2 c32_n = make_float2(0.f, 0.f);
            auto fetch = [&](int at) {
                ent_n = lists[at];
                nd_n = tnode[ent_n.x];
                m_n = mass[ent_n.x];
                if (MIXED) {
                    R_n = sscale[ent_n.x];
                    if (lane < P) c32_n = sexp[(size_t)ent_n.x * P + lane];
                } else if (lane < P) {
                    const double *ex = exps + (size_t)ent_n.x * 2 * P;
                    cr_n = ex[lane];
                    ci_n = ex[P + lane];
                }
            };
            if (b0 < e0) fetch(b0);
            for (int it = b0; it < e0; ++it) {
                const int2 ent = ent_n;
                const TNode nd = nd_n;
                const double mm = m_n;
                const float R = R_n;
                __syncwarp();
                if (lane < P) {
                    if (MIXED) {
                        float *cp = reinterpret_cast<float *>(s_coef32[warp]);
                        cp[4 * (lane >> 1) + (lane & 1)] = c32_n.x;
                        cp[4 * (lane >> 1) + 2 + (lane & 1)] = c32_n.y;
                    }
                    else s_coef[warp][lane] = {cr_n, ci_n};
                }
                __syncwarp();
                if (it + 1 < e0) fetch(it + 1);
                if ((ent.y >> lane) & 1) {
                    const double rz = x - nd.xcom, iz = y - nd.ycom;
                    const double r2 = rz * rz + iz * iz;
                    if (MIXED) {
                        // series: Re(u' Q(u')), u' = R / z, Q(u') = sum_j D_j u'^j
                        const float zr = (float)rz, zi = (float)iz;
                        const float inv = rcp_approx(zr * zr + zi * zi);
                        const float ur = R * zr * inv, ui = -R * zi * inv;
                        // Q(u') = E(w) + u' O(w), w = u'^2, E and O the even and odd parts
                        // of the series, evaluated together by Horner in f32x2 lanes
                        const float wr = fmaf(ur, ur, -ui * ui), wi = 2.f * ur * ui;
                        const float2 wr2 = make_float2(wr, wr), wi2 = make_float2(wi, wi);
                        const float2 nwi2 = make_float2(-wi, -wi);
                        const float4 cl = s_coef32[warp][P / 2 - 1];
                        float2 qr2 = make_float2(cl.x, cl.y), qi2 = make_float2(cl.z, cl.w);
#pragma unroll
                        for (int j = P / 2 - 2; j >= 0; --j) {
                            const float4 d = s_coef32[warp][j];
                            const float2 tr = __ffma2_rn(qi2, nwi2, make_float2(d.x, d.y));
                            const float2 ti = __ffma2_rn(qi2, wr2, make_float2(d.z, d.w));
                            const float2 nqr = __ffma2_rn(qr2, wr2, tr);
                            qi2 = __ffma2_rn(qr2, wi2, ti);
                            qr2 = nqr;
                        }
                        const float2 q = make_float2(
                            qr2.x + fmaf(ur, qr2.y, -ui * qi2.y),
                            qi2.x + fmaf(ur, qi2.y, ui * qr2.y));
                        two_sum_add(sh, sl, ur * q.x - ui * q.y);
                        far += mm * log_pos(r2, s_neg_log_c) * 0.5;
                    } else {
                        const double inv = 1.0 / r2;
                        const cplx u = {rz * inv, -iz * inv};
                        cplx q = s_coef[warp][P - 1];
#pragma unroll
                        for (int k = P - 2; k >= 0; --k) q = cfma(q, u, s_coef[warp][k]);
                        far += mm * log_pos(r2, s_neg_log_c) * 0.5 +
                               (u.re * q.re - u.im * q.im);
                    }
                }
            }
            if (MIXED) far += (double)sh + (double)sl;
        }

        // P2P (potential-kernels.m4:19-57): 0.5 sum v log(r2 + eps), sources
        // [part * PT_SEG, (part + 1) * PT_SEG) of the group's listed leaves.  Tiles of up to
        // PE_CHUNK consecutive sources of one leaf; the next tile is loaded into registers while
        // the current one is evaluated.
        {
            const int b1 = offs[ngroups + g], e1 = offs[ngroups + g + 1];
            int it = b1, skip = part * PT_SEG, budget = PT_SEG;
            int s_next = 0, e_next = 0;
            unsigned mask_next = 0;
            while (it < e1) {
                const int2 ent = lists[it++];
                const int2 rg = range[ent.x];
                const int cnt = rg.y - rg.x;
                if (skip < cnt) {
                    s_next = rg.x + skip;
                    e_next = rg.y;
                    mask_next = (unsigned)ent.y;
                    break;
                }
                skip -= cnt;
            }
            auto next_tile = [&](int &t0, int &tn, unsigned &msk) {
                while (s_next >= e_next && it < e1) {
                    const int2 ent = lists[it++];
                    const int2 rg = range[ent.x];
                    s_next = rg.x;
                    e_next = rg.y;
                    mask_next = (unsigned)ent.y;
                }
                t0 = s_next;
                tn = min(min(PE_CHUNK, e_next - s_next), budget);
                if (tn < 0) tn = 0;
                msk = mask_next;
                s_next += tn;
                budget -= tn;
            };
            int t0, tn;
            unsigned msk;
            next_tile(t0, tn, msk);
            double px = 0, py = 0, pv = 0;
            if (lane < tn) {
                px = xs[t0 + lane];
                py = ys[t0 + lane];
                pv = vs[t0 + lane];
            }
            float nh = 0, nl = 0, txh = 0, txl = 0, tyh = 0, tyl = 0;
            if (MIXED) {
                split2(x - xref, txh, txl);
                split2(y - yref, tyh, tyl);
            }
            const float ln2 = 0.6931471805599453f, epsf = (float)eps;
            while (tn > 0) {
                const int cnt = tn;
                const unsigned cmask = msk;   // this tile's targets (msk moves on to the next tile)
                const bool mine = (cmask >> lane) & 1;
                __syncwarp();
                if (MIXED) {
                    // source `lane` to entry lane / 2, half lane % 2; lanes past the tile add a
                    // zero-valued source at the reference point (finite, contributes 0)
                    float a = 0.f, b2 = 0.f, c2 = 0.f, d2 = 0.f, vv = 0.f;
                    if (lane < cnt) {
                        split2(px - xref, a, b2);
                        split2(py - yref, c2, d2);
                        vv = (float)pv;
                    }
                    float *nx = reinterpret_cast<float *>(s_nx[warp]);
                    float *ny = reinterpret_cast<float *>(s_ny[warp]);
                    const int e = 4 * (lane >> 1) + (lane & 1);
                    nx[e] = -a;
                    nx[e + 2] = -b2;
                    ny[e] = -c2;
                    ny[e + 2] = -d2;
                    reinterpret_cast<float *>(s_v2[warp])[lane] = vv;
                } else if (lane < cnt) {
                    s_xy[warp][lane] = make_double2(px, py);
                    s_v[warp][lane] = pv;
                }
                __syncwarp();
                next_tile(t0, tn, msk);
                if (lane < tn) {
                    px = xs[t0 + lane];
                    py = ys[t0 + lane];
                    pv = vs[t0 + lane];
                }
                // A tile needed by few targets of the group (k <= 16; k <= 8 in the mixed form,
                // whose per-pair cost is lower) is spread over the lanes:
                // lane l takes target q = l % k of the mask and sources l / k, l / k + r, ...
                // (r = 32 / k), and each target adds its r lane partials in lane order.  Denser
                // tiles keep one target per lane.
                const int k = __popc(cmask);
                if (k > (MIXED ? 8 : 16)) {
                    if (mine) {
                        if (MIXED) {
                            // two sources per step in f32x2 lanes; even and odd sources are
                            // summed apart and added at the end of the tile
                            const float2 txh2 = make_float2(txh, txh), txl2 = make_float2(txl, txl);
                            const float2 tyh2 = make_float2(tyh, tyh), tyl2 = make_float2(tyl, tyl);
                            const float2 eps2 = make_float2(epsf, epsf);
                            float2 acc = make_float2(0.f, 0.f);
                            const int npairs = (cnt + 1) >> 1;
#pragma unroll 4
                            for (int q = 0; q < npairs; ++q) {
                                const float4 nx = s_nx[warp][q], ny = s_ny[warp][q];
                                const float2 dx = __fadd2_rn(__fadd2_rn(txh2, make_float2(nx.x, nx.y)),
                                                             __fadd2_rn(txl2, make_float2(nx.z, nx.w)));
                                const float2 dy = __fadd2_rn(__fadd2_rn(tyh2, make_float2(ny.x, ny.y)),
                                                             __fadd2_rn(tyl2, make_float2(ny.z, ny.w)));
                                const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, eps2));
                                acc = __ffma2_rn(make_float2(lg2_approx(r2.x), lg2_approx(r2.y)),
                                                 s_v2[warp][q], acc);
                            }
                            two_sum_add(nh, nl, (acc.x + acc.y) * ln2);
                        } else {
#pragma unroll 4
                            for (int q = 0; q < cnt; ++q) {
                                const double2 sp = s_xy[warp][q];
                                const double xr = x - sp.x, yr = y - sp.y;
                                near += log_pos(fma(xr, xr, fma(yr, yr, eps)), s_neg_log_c) *
                                        s_v[warp][q];
                            }
                        }
                    }
                } else if (k > 0) {
                    const int r = 32 / k;
                    const int qt = lane % k;
                    const int tl = (int)__fns(cmask, 0, qt + 1);   // lane of this lane's target
                    double part = 0;
                    if (MIXED) {
                        const float qxh = __shfl_sync(FULL_MASK, txh, tl);
                        const float qxl = __shfl_sync(FULL_MASK, txl, tl);
                        const float qyh = __shfl_sync(FULL_MASK, tyh, tl);
                        const float qyl = __shfl_sync(FULL_MASK, tyl, tl);
                        float acc = 0;
                        const float *nx = reinterpret_cast<const float *>(s_nx[warp]);
                        const float *ny = reinterpret_cast<const float *>(s_ny[warp]);
                        const float *sv = reinterpret_cast<const float *>(s_v2[warp]);
                        if (lane < r * k)
                            for (int q = lane / k; q < cnt; q += r) {
                                const int e = 4 * (q >> 1) + (q & 1);
                                const float dx = (qxh + nx[e]) + (qxl + nx[e + 2]);
                                const float dy = (qyh + ny[e]) + (qyl + ny[e + 2]);
                                acc = fmaf(lg2_approx(fmaf(dx, dx, fmaf(dy, dy, epsf))), sv[q], acc);
                            }
                        part = (double)acc;
                    } else {
                        const double qx = __shfl_sync(FULL_MASK, x, tl);
                        const double qy = __shfl_sync(FULL_MASK, y, tl);
                        if (lane < r * k)
                            for (int q = lane / k; q < cnt; q += r) {
                                const double2 sp = s_xy[warp][q];
                                const double xr = qx - sp.x, yr = qy - sp.y;
                                part += log_pos(fma(xr, xr, fma(yr, yr, eps)), s_neg_log_c) *
                                        s_v[warp][q];
                            }
                    }
                    s_part[warp][lane] = part;
                    __syncwarp();
                    if (mine) {
                        const int q = __popc(cmask & ((1u << lane) - 1u));
                        double sum = 0;
                        for (int i = 0; i < r; ++i) sum += s_part[warp][q + i * k];
                        if (MIXED) two_sum_add(nh, nl, (float)sum * ln2);
                        else near += sum;
                    }
                    __syncwarp();
                }
            }
            if (MIXED) near = (double)nh + (double)nl;
        }
        const double res = 0.5 * near + far;
        if (nparts == 1) {
            if (valid) out[j] = res;
        } else {
            partial[(size_t)task * 32 + lane] = res;
        }
        __syncwarp();
    }
}

__global__ void k_task_map_groups(int ngroups, const int *__restrict__ offs,
                                  int *__restrict__ task_group) {
    const int *toff = offs + 2 * ngroups;
    const int tbase = toff[0];
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gridDim.x * blockDim.x)
        for (int t = toff[g]; t < toff[g + 1]; ++t) task_group[t - tbase] = g;
}

// Sum of the parts of every multi-task group, in task order (deterministic).
__global__ void k_potential_gather_parts(int ngroups, int m, const int *__restrict__ tperm,
                                         const int *__restrict__ offs,
                                         const double *__restrict__ partial,
                                         double *__restrict__ out) {
    const int lane = lane_id();
    const int *toff = offs + 2 * ngroups;
    const int tbase = toff[0];
    for (int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < ngroups;
         g += (gridDim.x * blockDim.x) >> 5) {
        const int t0 = toff[g] - tbase, np = toff[g + 1] - toff[g];
        if (np <= 1) continue;
        double s = 0;
        for (int p = 0; p < np; ++p) s += partial[(size_t)(t0 + p) * 32 + lane];
        const int t = g * 32 + lane;
        if (t < m) out[tperm[t]] = s;
    }
}

// Mixed form: a_k / R^(k+1) in FP32, R = the cell's power-of-two radius (see force.cu).
template <int P>
__global__ void k_scale_coeffs_pot(int nnodes, const TNode *__restrict__ tnode,
                                   const double *__restrict__ exps, float2 *__restrict__ sexp,
                                   float *__restrict__ sscale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)nnodes * P;
         i += (long long)gridDim.x * blockDim.x) {
        const int node = (int)(i / P), k = (int)(i % P);
        const double r = tnode[node].r;
        int e = 0;
        if (r > 0 && r < 1e300) frexp(r, &e);
        const double *ex = exps + (size_t)node * 2 * P;
        sexp[i] = make_float2((float)ldexp(ex[k], -e * (k + 1)), (float)ldexp(ex[P + k], -e * (k + 1)));
        if (k == 0) sscale[node] = (float)ldexp(1.0, e);
    }
}

static int sm_count_p() { return device_sm_count(); }

// Target sort and lists run on the auxiliary stream; `between` (the expansion work) runs on the
// main stream meanwhile, and the evaluation waits for both.
int potential(Context &c, double theta, const double *xt, const double *yt, int m, double *out,
              OverlapFn between) {
    if (m == 0) return between ? between(c) : TC_OK;
    int rc;
    int *tkeys, *tperm, *tkeys2, *tperm2;
    if ((rc = ensure(c, S_TKEYS, m, &tkeys)) || (rc = ensure(c, S_TPERM, m, &tperm)) ||
        (rc = ensure(c, S_TKEYS2, m, &tkeys2)) || (rc = ensure(c, S_TPERM2, m, &tperm2)))
        return rc;
    const int ngroups = (m + 31) / 32;
    // counts / offsets: E2P | P2P list lengths and evaluation tasks, ngroups each
    int *counts, *offs;
    if ((rc = ensure(c, S_PCOUNT, (size_t)3 * ngroups, &counts)) ||
        (rc = ensure(c, S_POFF, (size_t)3 * ngroups + 1, &offs)))
        return rc;
    const TNode *tnode = slot_ptr<TNode>(c, S_TNODE);
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);
    const int grid = (int)std::min<long long>((ngroups + PT_WARPS - 1) / PT_WARPS,
                                              (long long)sm_count_p() * 16);
    int *ko, *vo;
    // One walk counts the lists and writes them into per-warp scratch runs; after the scan a
    // copy puts them in CSR order.  If a run outgrew its region a second walk writes them
    // instead, and the regions are sized up for the next solve.  The runs live in the sort's
    // record buffer when they fit in it, else in a block held only for the build.
    const int nwarps = grid * PT_WARPS;
    ScratchLayout sl;
    ListScratch ls;   // released (when transient) after the copy, in stream order
    int *sstart, *meta;
    unsigned long long *stats = slot_ptr<unsigned long long>(c, S_STATS);
    TC_CUDA_TRY(cudaEventRecord(c.ev_fork, c.stream));
    {
        AuxScope on_aux(c);
        TC_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.ev_fork, 0));
        if ((rc = target_keys(c, xt, yt, m, tkeys, nullptr))) return rc;
        if ((rc = radix_sort_pairs(c, tkeys, nullptr, m, 2 * LMAX, tkeys2, tperm2, tkeys, tperm,
                                   &ko, &vo)))
            return rc;
        if ((rc = list_scratch(c, 2, nwarps, ngroups, sizeof(int2), sl, ls)) ||
            (rc = ensure(c, S_LSTART, (size_t)2 * ngroups, &sstart)) ||
            (rc = ensure(c, S_LMETA, 4, &meta)))
            return rc;
        TC_CUDA_TRY(cudaMemsetAsync(meta, 0, sizeof(int) * 4, c.stream));
        k_potential_lists<2><<<grid, PT_WARPS * 32, 0, c.stream>>>(
            ngroups, m, xt, yt, vo, theta, tnode, c.nnodes, counts, nullptr, nullptr,
            static_cast<int2 *>(ls.p), sl, sstart, meta, err, stats);
        TC_KERNEL_CHECK();
        if ((rc = exclusive_scan(c, counts, offs, 3 * ngroups))) return rc;
        for (int k = 0; k < 3; ++k)
            TC_CUDA_TRY(cudaMemcpyAsync(c.h_pinned + 32 + k, offs + (k + 1) * ngroups, sizeof(int),
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
    const int n_e2p = (int)c.h_pinned[32], total = (int)c.h_pinned[33];
    const int ntasks = (int)c.h_pinned[34] - total;
    const bool overflow = c.h_pinned[36] != 0;
    c.list_walks = overflow ? 2 : 1;
    scratch_learn(c, 2, nwarps, ngroups, c.h_pinned + 37);   // for the next solve
    c.counts.n_e2p = n_e2p;
    c.counts.n_p2p = total - n_e2p;
    c.counts.n_e2l = 0;
    c.counts.e2l_pairs = 0;
    c.counts.l2p_targets = 0;
    int2 *lists;
    {
        AuxScope on_aux(c);
        if ((rc = ensure(c, S_PE2P, (size_t)total + 1, &lists))) return rc;
        if (!overflow) {
            k_potential_lists_copy<<<(int)std::min<long long>((ngroups + 7) / 8,
                                                              (long long)sm_count_p() * 16),
                                     256, 0, c.stream>>>(ngroups, counts, offs, sstart,
                                                         static_cast<const int2 *>(ls.p), lists);
        } else {
            // the second walk adds the work counters again: clear the first walk's
            TC_CUDA_TRY(cudaMemsetAsync(stats + STAT_E2P_PAIRS, 0, 2 * sizeof(unsigned long long),
                                        c.stream));
            k_potential_lists<1><<<grid, PT_WARPS * 32, 0, c.stream>>>(
                ngroups, m, xt, yt, vo, theta, tnode, c.nnodes, nullptr, offs, lists, nullptr,
                sl, nullptr, nullptr, err, stats);
        }
        TC_KERNEL_CHECK();
        TC_CUDA_TRY(cudaEventRecord(c.ev_join, c.stream));
    }
    TC_CUDA_TRY(cudaStreamWaitEvent(c.stream, c.ev_join, 0));
    phase_mark(c, 4);
    int *task_ctr, *task_group;
    double *partial;
    if ((rc = ensure(c, S_BRICK_CTR, 4, &task_ctr)) ||
        (rc = ensure(c, S_TASKMAP, (size_t)ntasks, &task_group)) ||
        (rc = ensure(c, S_FPART, (size_t)ntasks * 32, &partial)))
        return rc;
    TC_CUDA_TRY(cudaMemsetAsync(task_ctr, 0, sizeof(int), c.stream));
    k_task_map_groups<<<(int)std::min<long long>((ngroups + 255) / 256, (long long)sm_count_p() * 8),
                        256, 0, c.stream>>>(ngroups, offs, task_group);
    TC_KERNEL_CHECK();
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
            k_scale_coeffs_pot<P>
                <<<(int)std::min<long long>((items + 255) / 256, (long long)sm_count_p() * 8), 256, 0,
                   c.stream>>>(c.nnodes, tnode, slot_ptr<double>(c, S_EXPS), sexp, sscale);
            TC_KERNEL_CHECK();
        }
        auto eval = mixed ? k_potential_eval<P, true> : k_potential_eval<P, false>;
        const int occ = mixed ? blocks_per_sm<k_potential_eval<P, true>>(PE_WARPS * 32, 0)
                              : blocks_per_sm<k_potential_eval<P, false>>(PE_WARPS * 32, 0);
        const int egrid = (int)std::min<long long>((ntasks + PE_WARPS - 1) / PE_WARPS,
                                                   (long long)sm_count_p() * occ);
        phase_mark(c, 6);
        eval<<<egrid, PE_WARPS * 32, 0, c.stream>>>(
            ngroups, m, xt, yt, vo, tnode, slot_ptr<double>(c, S_MASS), slot_ptr<double>(c, S_EXPS),
            slot_ptr<int2>(c, S_RANGE), slot_ptr<double>(c, S_XS), slot_ptr<double>(c, S_YS),
            slot_ptr<double>(c, S_VS), offs, lists, out, partial, task_ctr, task_group, sexp, sscale);
        TC_KERNEL_CHECK();
        return TC_OK;
    });
    if (rc) return rc;
    phase_mark(c, 7);
    if (ntasks > ngroups) {
        k_potential_gather_parts<<<(int)std::min<long long>((ngroups + 7) / 8, (long long)sm_count_p() * 16),
                                   256, 0, c.stream>>>(ngroups, m, vo, offs, partial, out);
        TC_KERNEL_CHECK();
    }
    return TC_OK;
}

void kernels_potential(KernelList &v) {
    v.insert(v.end(), {(const void *)k_potential_lists<1>, (const void *)k_potential_lists<2>,
                       (const void *)k_potential_lists_copy, (const void *)k_task_map_groups,
                       (const void *)k_potential_gather_parts});
#define TC_POTENTIAL_KERNELS(P)                                                                  \
    v.insert(v.end(), {(const void *)k_potential_eval<P, true>,                                 \
                       (const void *)k_potential_eval<P, false>, (const void *)k_scale_coeffs_pot<P>});
    TC_FOR_EACH_ORDER(TC_POTENTIAL_KERNELS)
#undef TC_POTENTIAL_KERNELS
}

}  // namespace tc
