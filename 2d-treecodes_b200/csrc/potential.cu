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
constexpr int PT_STACK = 64;   // depth-first, one entry popped per step: <= 3 * LMAX + 4 live entries

template <bool FILL>
__global__ __launch_bounds__(PT_WARPS * 32) void k_potential_lists(
    int ngroups, int m, const double *__restrict__ xt, const double *__restrict__ yt,
    const int *__restrict__ tperm, double theta, const TNode *__restrict__ tnode, int nnodes,
    int *__restrict__ counts, const int *__restrict__ offs, int2 *__restrict__ lists,
    unsigned *err, unsigned long long *stats) {
    __shared__ int2 stack_all[PT_WARPS][PT_STACK];
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    int2 *stack = stack_all[warp];
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
        int o0 = 0, o1 = 0, l0 = 0, l1 = 0;
        if (FILL) {
            o0 = offs[g];
            l0 = offs[g + 1];
            o1 = offs[ngroups + g];
            l1 = offs[ngroups + g + 1];
        }
        int n0 = 0, n1 = 0;
        int top = 0;
        if (lane == 0) stack[0] = make_int2(0, (int)vmask);
        top = 1;
        __syncwarp();
        while (top > 0) {
            --top;
            const int2 ent = stack[top];
            __syncwarp();
            const unsigned mask = (unsigned)ent.y;
            if ((unsigned)ent.x >= (unsigned)nnodes) {
                if (lane == 0) atomicOr(err, DEVERR_BOUNDS);
                continue;
            }
            const TNode nd = tnode[ent.x];
            // r2 = (xt - xcom)^2 + (yt - ycom)^2 without contraction, as the compiled reference
            const double dx = __dsub_rn(x, nd.xcom), dy = __dsub_rn(y, nd.ycom);
            const double r2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
            const bool accept = ((mask >> lane) & 1u) && __dmul_rn(nd.r, nd.r) < __dmul_rn(theta2, r2);
            const unsigned far = __ballot_sync(FULL_MASK, accept);
            const unsigned rest = mask & ~far;
            if (far) {
                e2p_pairs += __popc(far);
                if (FILL && lane == 0) {
                    if (o0 + n0 < l0) lists[o0 + n0] = make_int2(ent.x, (int)far);
                    else atomicOr(err, DEVERR_BOUNDS);
                }
                ++n0;
            }
            if (rest) {
                if (nd.child < 0) {
                    if (nd.count > 0) {
                        p2p_pairs += (unsigned long long)__popc(rest) * (unsigned)nd.count;
                        if (FILL && lane == 0) {
                            if (o1 + n1 < l1) lists[o1 + n1] = make_int2(ent.x, (int)rest);
                            else atomicOr(err, DEVERR_BOUNDS);
                        }
                        ++n1;
                    }
                } else {
                    if (nd.child <= ent.x || nd.child + 4 > nnodes) {
                        if (lane == 0) atomicOr(err, DEVERR_BOUNDS);
                        continue;
                    }
                    if (top + 4 > PT_STACK) {
                        if (lane == 0) atomicOr(err, DEVERR_STACK);
                        break;
                    }
                    if (lane < 4) stack[top + lane] = make_int2(nd.child + 3 - lane, (int)rest);
                    top += 4;
                }
            }
            __syncwarp();
        }
        if (!FILL && lane == 0) {
            counts[g] = n0;
            counts[ngroups + g] = n1;
        }
        __syncwarp();
    }
    if (FILL && lane == 0) {
        if (e2p_pairs) atomicAdd(&stats[STAT_E2P_PAIRS], e2p_pairs);
        if (p2p_pairs) atomicAdd(&stats[STAT_P2P_PAIRS], p2p_pairs);
    }
}

constexpr int PE_WARPS = 4;
constexpr int PE_CHUNK = 32;

template <int P>
__global__ __launch_bounds__(PE_WARPS * 32) void k_potential_eval(
    int ngroups, int m, const double *__restrict__ xt, const double *__restrict__ yt,
    const int *__restrict__ tperm, const TNode *__restrict__ tnode,
    const double *__restrict__ mass, const double *__restrict__ exps,
    const int2 *__restrict__ range, const double *__restrict__ xs,
    const double *__restrict__ ys, const double *__restrict__ vs,
    const int *__restrict__ offs, const int2 *__restrict__ lists, double *__restrict__ out) {
    __shared__ cplx s_coef[PE_WARPS][P];
    __shared__ double2 s_xy[PE_WARPS][PE_CHUNK];
    __shared__ double s_v[PE_WARPS][PE_CHUNK];
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    const double eps = 10 * DBL_EPSILON;

    for (int g = blockIdx.x * PE_WARPS + warp; g < ngroups; g += gridDim.x * PE_WARPS) {
        const int t = g * 32 + lane;
        const bool valid = t < m;
        int j = 0;
        double x = 0, y = 0;
        if (valid) {
            j = tperm[t];
            x = xt[j];
            y = yt[j];
        }
        double far = 0, near = 0;

        // E2P (potential-kernels.m4:59-89): m log(r2)/2 + Re sum_{j=1..p} a_{j-1} z^-j
        const int b0 = offs[g], e0 = offs[g + 1];
        for (int it = b0; it < e0; ++it) {
            const int2 ent = lists[it];
            const TNode nd = tnode[ent.x];
            const double mm = mass[ent.x];
            __syncwarp();
            if (lane < P) {
                const double *ex = exps + (size_t)ent.x * 2 * P;
                s_coef[warp][lane] = {ex[lane], ex[P + lane]};
            }
            __syncwarp();
            if ((ent.y >> lane) & 1) {
                const double rz = x - nd.xcom, iz = y - nd.ycom;
                const double r2 = rz * rz + iz * iz;
                const double inv = 1.0 / r2;
                const cplx u = {rz * inv, -iz * inv};
                cplx q = s_coef[warp][P - 1];
#pragma unroll
                for (int k = P - 2; k >= 0; --k) q = cfma(q, u, s_coef[warp][k]);
                far += mm * log(r2) * 0.5 + (u.re * q.re - u.im * q.im);
            }
        }

        // P2P (potential-kernels.m4:19-57): 0.5 sum v log(r2 + eps)
        const int b1 = offs[ngroups + g], e1 = offs[ngroups + g + 1];
        for (int it = b1; it < e1; ++it) {
            const int2 ent = lists[it];
            const int2 rg = range[ent.x];
            const bool mine = (ent.y >> lane) & 1;
            for (int s0 = rg.x; s0 < rg.y; s0 += PE_CHUNK) {
                const int cnt = min(PE_CHUNK, rg.y - s0);
                __syncwarp();
                if (lane < cnt) {
                    s_xy[warp][lane] = make_double2(xs[s0 + lane], ys[s0 + lane]);
                    s_v[warp][lane] = vs[s0 + lane];
                }
                __syncwarp();
                if (mine) {
                    for (int k = 0; k < cnt; ++k) {
                        const double2 sp = s_xy[warp][k];
                        const double xr = x - sp.x, yr = y - sp.y;
                        near += log(xr * xr + yr * yr + eps) * s_v[warp][k];
                    }
                }
            }
        }
        if (valid) out[j] = 0.5 * near + far;
        __syncwarp();
    }
}

static int sm_count_p() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

int potential(Context &c, double theta, const double *xt, const double *yt, int m, double *out) {
    if (c.order != ORDER_POTENTIAL) {
        set_error(TC_ERR_INVALID, "potential evaluation needs an order-%d tree", ORDER_POTENTIAL);
        return TC_ERR_INVALID;
    }
    if (m == 0) return TC_OK;
    int rc;
    int *tkeys, *tperm, *tkeys2, *tperm2;
    if ((rc = ensure(c, S_TKEYS, m, &tkeys)) || (rc = ensure(c, S_TPERM, m, &tperm)) ||
        (rc = ensure(c, S_TKEYS2, m, &tkeys2)) || (rc = ensure(c, S_TPERM2, m, &tperm2)))
        return rc;
    if ((rc = target_keys(c, xt, yt, m, tkeys, nullptr))) return rc;
    int *ko, *vo;
    if ((rc = radix_sort_pairs(c, tkeys, nullptr, m, 2 * LMAX, tkeys2, tperm2, tkeys, tperm, &ko, &vo)))
        return rc;
    const int ngroups = (m + 31) / 32;
    int *counts, *offs;
    if ((rc = ensure(c, S_PCOUNT, (size_t)2 * ngroups, &counts)) ||
        (rc = ensure(c, S_POFF, (size_t)2 * ngroups + 1, &offs)))
        return rc;
    const TNode *tnode = slot_ptr<TNode>(c, S_TNODE);
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);
    const int grid = (int)std::min<long long>((ngroups + PT_WARPS - 1) / PT_WARPS,
                                              (long long)sm_count_p() * 16);
    k_potential_lists<false><<<grid, PT_WARPS * 32, 0, c.stream>>>(ngroups, m, xt, yt, vo, theta,
                                                                  tnode, c.nnodes, counts, nullptr, nullptr,
                                                                  err, nullptr);
    TC_KERNEL_CHECK();
    if ((rc = exclusive_scan(c, counts, offs, 2 * ngroups))) return rc;
    TC_CUDA_TRY(cudaMemcpyAsync(c.h_pinned, offs + ngroups, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    TC_CUDA_TRY(cudaMemcpyAsync(c.h_pinned + 1, offs + 2 * ngroups, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    TC_CUDA_TRY(cudaStreamSynchronize(c.stream));
    const int n_e2p = (int)c.h_pinned[0], total = (int)c.h_pinned[1];
    c.counts.n_e2p = n_e2p;
    c.counts.n_p2p = total - n_e2p;
    c.counts.n_e2l = 0;
    c.counts.e2l_pairs = 0;
    c.counts.l2p_targets = 0;
    int2 *lists;
    if ((rc = ensure(c, S_PE2P, (size_t)total + 1, &lists))) return rc;
    k_potential_lists<true><<<grid, PT_WARPS * 32, 0, c.stream>>>(ngroups, m, xt, yt, vo, theta,
                                                                 tnode, c.nnodes, nullptr, offs, lists, err,
                                                                 slot_ptr<unsigned long long>(c, S_STATS));
    TC_KERNEL_CHECK();
    phase_mark(c, 4);
    const int egrid = (int)std::min<long long>((ngroups + PE_WARPS - 1) / PE_WARPS,
                                               (long long)sm_count_p() * 8);
    k_potential_eval<ORDER_POTENTIAL><<<egrid, PE_WARPS * 32, 0, c.stream>>>(
        ngroups, m, xt, yt, vo, tnode, slot_ptr<double>(c, S_MASS), slot_ptr<double>(c, S_EXPS),
        slot_ptr<int2>(c, S_RANGE), slot_ptr<double>(c, S_XS), slot_ptr<double>(c, S_YS),
        slot_ptr<double>(c, S_VS), offs, lists, out);
    TC_KERNEL_CHECK();
    return TC_OK;
}

}  // namespace tc
