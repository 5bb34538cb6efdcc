// upward.cu -- leaf setup + P2E and the E2E climb, in one kernel.
//
// One warp per leaf (drivers/upward.cpp:61-93, kernels/upward-common.ispc:13-57,
// kernels/upward-kernels.m4:18-93).  After writing its leaf, the warp increments the parent's
// arrival counter; the warp that brings it to four merges the four children and shifts their
// expansions into the parent (upward.cpp:95-218, kernels/upward-kernels.m4:95-149), then climbs
// on.  No per-level launches are needed; children's data written by other warps is read with
// L2-coherent loads (__ldcg) after a device-scope fence.
//
// Bit-exact restatements (decisions of the traversals depend on these values):
//  * leaf mass / |v| weights / weighted sums: four strided lane accumulators, reduced as
//    (l0 + l1) + (l2 + l3); a lane whose own weight sum is zero measures the radius about the
//    origin (upward-common.ispc:44-45 tests the varying wsum);
//  * leaf com = wx/w, or the cell centre fma(0.5, h, fma(cx, h, xmin)) when w == 0;
//  * parent sums over children as (c0 + c3) + (c1 + c2), the order the compiled driver uses;
//  * parent radius min(max_c (sqrt(fma(rx, rx, ry*ry)) + r_c), (double)1.4143f * ext / 2^l)
//    over children with nonzero weight;
//  * when all four children are negligible (|w| < 1.1e-16) the parent's expansion is zeroed and
//    child 3 -- the last child to arrive in the reference's sequential subtree order -- becomes
//    an empty leaf (upward.cpp:173-180); with exactly three negligible children the remaining
//    child's coefficients are copied unshifted (upward.cpp:182-188).
//
// Expansion layout: exps[node][0][k] real parts, exps[node][1][k] imaginary parts, k < ORDER.
#include "tc_internal.h"
#include "tc_math.cuh"

namespace tc {

__constant__ BinomTable c_binom_up = make_binom_table();

constexpr int UP_WARPS = 4;
constexpr int UP_CHUNK = 256;   // leaf sources staged in shared memory per pass (multiple of 4)

template <int P>
struct UpShared {
    double zr[4][P + 1], zi[4][P + 1];   // z0^-k per child
    double cr[4][P + 1], ci[4][P + 1];   // a_{k-1} z0^-k per child
    double sx[UP_CHUNK], sy[UP_CHUNK], sv[UP_CHUNK];   // staged leaf sources
};

template <int P>
__device__ void shift_children(UpShared<P> &sh, const double *exps, int cb, const double *cm,
                               const double *cx, const double *cy, double px, double py,
                               double *dst) {
    const int lane = lane_id();
    if (lane < 4) {
        const int c = lane;
        const double x0 = cx[c] - px, y0 = cy[c] - py;
        const double r2z0 = x0 * x0 + y0 * y0;
        const double rinv = x0 / r2z0, iinv = -y0 / r2z0;
        double zr = rinv, zi = iinv;
        sh.zr[c][1] = zr;
        sh.zi[c][1] = zi;
        for (int j = 2; j <= P; ++j) {
            const double tr = zr * rinv - zi * iinv;
            const double ti = zr * iinv + zi * rinv;
            zr = tr;
            zi = ti;
            sh.zr[c][j] = zr;
            sh.zi[c][j] = zi;
        }
    }
    __syncwarp();
    for (int it = lane; it < 4 * P; it += 32) {
        const int c = it / P, k = it % P + 1;
        const double *ex = exps + (size_t)(cb + c) * 2 * P;
        const double ar = __ldcg(ex + k - 1), ai = __ldcg(ex + P + k - 1);
        sh.cr[c][k] = ar * sh.zr[c][k] - ai * sh.zi[c][k];
        sh.ci[c][k] = ar * sh.zi[c][k] + ai * sh.zr[c][k];
    }
    __syncwarp();
    if (lane < P) {
        const int l = lane + 1;
        const double minv = -1.0 / l;
        double pr[4], pi[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            double rtmp = l == 1 ? -cm[c] : cm[c] * minv;
            double itmp = 0;
            for (int k = 1; k <= l; ++k) {
                const double b = c_binom_up.c[l - 1][k - 1];
                rtmp += sh.cr[c][k] * b;
                itmp += sh.ci[c][k] * b;
            }
            const double zr = sh.zr[c][l], zi = sh.zi[c][l];
            const double invz2 = zr * zr + zi * zi;
            const double inv = invz2 != 0 ? 1.0 / invz2 : 0.0;
            const double rz = zr * inv, iz = -zi * inv;
            pr[c] = rtmp * rz - itmp * iz;
            pi[c] = rtmp * iz + itmp * rz;
        }
        dst[l - 1] = (pr[0] + pr[1]) + (pr[2] + pr[3]);
        dst[P + l - 1] = (pi[0] + pi[1]) + (pi[2] + pi[3]);
    }
    __syncwarp();
}

template <int P>
__global__ __launch_bounds__(UP_WARPS * 32) void k_upward(
    int nnodes, int nsrc, int leafcap, const double *__restrict__ xs, const double *__restrict__ ys,
    const double *__restrict__ vs, const int2 *__restrict__ range, const int4 *__restrict__ cell,
    TNode *tnode, double *mass, double *wgt, double *wxs, double *wys, double *exps, int *upcnt,
    const Frame *__restrict__ frame, unsigned *err) {
    __shared__ UpShared<P> shared[UP_WARPS];
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    UpShared<P> &sh = shared[warp];
    const int node = blockIdx.x * UP_WARPS + warp;
    if (node >= nnodes) return;
    const int2 rg = range[node];
    const int4 cl = cell[node];
    const bool leaf = (rg.y - rg.x <= leafcap) || cl.x == LMAX;
    if (!leaf) return;
    if (rg.x < 0 || rg.y < rg.x || rg.y > nsrc || cl.w >= nnodes || cl.x < 0 || cl.x > LMAX) {
        if (lane == 0) atomicOr(err, DEVERR_BOUNDS);
        return;
    }
    const Frame f = *frame;
    const int s = rg.x, e = rg.y;

    // Leaf sources pass through shared memory in chunks of UP_CHUNK (coalesced loads by all
    // lanes); a leaf that fits one chunk is loaded once for all three passes below.
    const int nch = (e - s + UP_CHUNK - 1) / UP_CHUNK;
    auto stage = [&](int c0, int cnt) {
        __syncwarp();
        for (int j = lane; j < cnt; j += 32) {
            sh.sx[j] = xs[c0 + j];
            sh.sy[j] = ys[c0 + j];
            sh.sv[j] = vs[c0 + j];
        }
        __syncwarp();
    };

    // ---- upward_setup: four strided lane accumulators (upward-common.ispc:24-42); chunks
    // start at multiples of 4 from s, so element i still goes to lane (i - s) % 4.
    double ms = 0, ws = 0, wxs_l = 0, wys_l = 0;
    for (int ch = 0; ch < nch; ++ch) {
        const int c0 = s + ch * UP_CHUNK, cnt = min(UP_CHUNK, e - c0);
        stage(c0, cnt);
        if (lane < 4)
            for (int j = lane; j < cnt; j += 4) {
                const double x = sh.sx[j], y = sh.sy[j], m = sh.sv[j];
                const double w = fabs(m);
                ms = __dadd_rn(ms, m);
                ws = __dadd_rn(ws, w);
                wxs_l = __dadd_rn(wxs_l, __dmul_rn(x, w));
                wys_l = __dadd_rn(wys_l, __dmul_rn(y, w));
            }
    }
    auto reduce4 = [&](double v) {
        const double a = __dadd_rn(v, __shfl_down_sync(FULL_MASK, v, 1));   // lane0: l0+l1, lane2: l2+l3
        return __shfl_sync(FULL_MASK, __dadd_rn(a, __shfl_down_sync(FULL_MASK, a, 2)), 0);
    };
    const double msum = reduce4(ms);
    const double wsum = reduce4(ws);
    const double xsum = reduce4(wxs_l);
    const double ysum = reduce4(wys_l);

    // radius about the per-lane centre (upward-common.ispc:44-56)
    double r2 = 0;
    {
        const double lx = ws != 0 ? __ddiv_rn(xsum, wsum) : 0.0;
        const double ly = ws != 0 ? __ddiv_rn(ysum, wsum) : 0.0;
        for (int ch = 0; ch < nch; ++ch) {
            const int c0 = s + ch * UP_CHUNK, cnt = min(UP_CHUNK, e - c0);
            if (nch > 1) stage(c0, cnt);
            if (lane < 4)
                for (int j = lane; j < cnt; j += 4) {
                    const double xr = __dsub_rn(sh.sx[j], lx), yr = __dsub_rn(sh.sy[j], ly);
                    r2 = fmax(r2, __dadd_rn(__dmul_rn(xr, xr), __dmul_rn(yr, yr)));
                }
        }
    }
    r2 = fmax(r2, __shfl_down_sync(FULL_MASK, r2, 1));
    r2 = fmax(r2, __shfl_down_sync(FULL_MASK, r2, 2));
    const double radius = __dsqrt_rn(__shfl_sync(FULL_MASK, r2, 0));

    // com (upward.cpp:71-72; x0 = fma(cx, h, xmin) as in build_tree)
    double xcom, ycom;
    if (wsum != 0) {
        xcom = __ddiv_rn(xsum, wsum);
        ycom = __ddiv_rn(ysum, wsum);
    } else {
        const double h = __ddiv_rn(f.ext, (double)(1 << cl.x));
        xcom = __fma_rn(0.5, h, __fma_rn((double)cl.y, h, f.xmin));
        ycom = __fma_rn(0.5, h, __fma_rn((double)cl.z, h, f.ymin));
    }

    // ---- upward_p2e: a_n = -sum v (z - c)^(n+1) / (n+1)
    double ar[P], ai[P];
#pragma unroll
    for (int n = 0; n < P; ++n) ar[n] = ai[n] = 0;
    for (int ch = 0; ch < nch; ++ch) {
        const int c0 = s + ch * UP_CHUNK, cnt = min(UP_CHUNK, e - c0);
        if (nch > 1) stage(c0, cnt);
        for (int j = lane; j < cnt; j += 32) {
            const double r0 = sh.sx[j] - xcom, i0 = sh.sy[j] - ycom, src = sh.sv[j];
            double pr = r0, pim = i0;
            ar[0] -= r0 * src;
            ai[0] -= i0 * src;
#pragma unroll
            for (int n = 1; n < P; ++n) {
                const double tr = pr * r0 - pim * i0;
                const double ti = pr * i0 + pim * r0;
                pr = tr;
                pim = ti;
                const double term = src * (1.0 / (n + 1));
                ar[n] -= pr * term;
                ai[n] -= pim * term;
            }
        }
    }
#pragma unroll
    for (int n = 0; n < P; ++n) {
        for (int m = 16; m; m >>= 1) {
            ar[n] += shfl_xor_d(ar[n], m);
            ai[n] += shfl_xor_d(ai[n], m);
        }
    }
    double *ex = exps + (size_t)node * 2 * P;
#pragma unroll
    for (int n = 0; n < P; ++n)
        if (lane == (n & 31)) {
            ex[n] = ar[n];
            ex[P + n] = ai[n];
        }
    if (lane == 0) {
        tnode[node].xcom = xcom;
        tnode[node].ycom = ycom;
        tnode[node].r = radius;
        mass[node] = msum;
        wgt[node] = wsum;
        wxs[node] = xsum;
        wys[node] = ysum;
    }

    // ---- climb (upward.cpp:95-218)
    int parent = cl.w;
    while (parent >= 0) {
        __threadfence();
        __syncwarp();
        int prev = 0;
        if (lane == 0) prev = atomicAdd(&upcnt[parent], 1);
        prev = __shfl_sync(FULL_MASK, prev, 0);
        if (prev != 3) return;
        __threadfence();

        const int cb = __ldcg(&tnode[parent].child);
        const int plevel = cell[parent].x;
        if (cb <= parent || cb + 4 > nnodes) {
            if (lane == 0) atomicOr(err, DEVERR_BOUNDS);
            return;
        }
        double cm[4], cw[4], cwx[4], cwy[4], cxc[4], cyc[4], cr[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            cm[c] = __ldcg(&mass[cb + c]);
            cw[c] = __ldcg(&wgt[cb + c]);
            cwx[c] = __ldcg(&wxs[cb + c]);
            cwy[c] = __ldcg(&wys[cb + c]);
            cxc[c] = __ldcg(&tnode[cb + c].xcom);
            cyc[c] = __ldcg(&tnode[cb + c].ycom);
            cr[c] = __ldcg(&tnode[cb + c].r);
        }
        const double pm = __dadd_rn(__dadd_rn(cm[0], cm[3]), __dadd_rn(cm[1], cm[2]));
        const double pw = __dadd_rn(__dadd_rn(cw[0], cw[3]), __dadd_rn(cw[1], cw[2]));
        const double pwx = __dadd_rn(__dadd_rn(cwx[0], cwx[3]), __dadd_rn(cwx[1], cwx[2]));
        const double pwy = __dadd_rn(__dadd_rn(cwy[0], cwy[3]), __dadd_rn(cwy[1], cwy[2]));
        const double px = __ddiv_rn(pwx, pw), py = __ddiv_rn(pwy, pw);
        double rr = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (cw[c] != 0) {
                const double rx = __dsub_rn(px, cxc[c]), ry = __dsub_rn(py, cyc[c]);
                const double cand = __dadd_rn(__dsqrt_rn(__fma_rn(rx, rx, __dmul_rn(ry, ry))), cr[c]);
                rr = cand > rr ? cand : rr;
            }
        const double cap = __ddiv_rn(__dmul_rn((double)1.4143f, f.ext), (double)(1 << plevel));
        const double prad = cap < rr ? cap : rr;

        int zcount = 0, nz = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const bool negl = fabs(cw[c]) < 1.1e-16;
            zcount += negl;
            if (!negl) nz = c;
        }
        double *dst = exps + (size_t)parent * 2 * P;
        if (zcount == 4) {
            for (int k = lane; k < 2 * P; k += 32) dst[k] = 0.0;
            if (lane == 0) {
                tnode[cb + 3].child = -1;
                tnode[cb + 3].count = 0;
            }
        } else if (zcount == 3) {
            const double *src = exps + (size_t)(cb + nz) * 2 * P;
            for (int k = lane; k < 2 * P; k += 32) dst[k] = __ldcg(src + k);
        } else {
            shift_children<P>(sh, exps, cb, cm, cxc, cyc, px, py, dst);
        }
        if (lane == 0) {
            tnode[parent].xcom = px;
            tnode[parent].ycom = py;
            tnode[parent].r = prad;
            mass[parent] = pm;
            wgt[parent] = pw;
            wxs[parent] = pwx;
            wys[parent] = pwy;
        }
        parent = cell[parent].w;
        if (parent >= nnodes) {
            if (lane == 0) atomicOr(err, DEVERR_BOUNDS);
            return;
        }
    }
}

int upward_pass(Context &c, int order) {
    const int nn = c.nnodes;
    int rc;
    double *mass, *w, *wx, *wy, *exps;
    int *upcnt;
    if ((rc = ensure(c, S_MASS, nn, &mass)) || (rc = ensure(c, S_W, nn, &w)) ||
        (rc = ensure(c, S_WX, nn, &wx)) || (rc = ensure(c, S_WY, nn, &wy)) ||
        (rc = ensure(c, S_EXPS, (size_t)nn * 2 * order, &exps)) ||
        (rc = ensure(c, S_UPCNT, nn, &upcnt)))
        return rc;
    TC_CUDA_TRY(cudaMemsetAsync(upcnt, 0, sizeof(int) * nn, c.stream));
    const int grid = (nn + UP_WARPS - 1) / UP_WARPS;
    const double *xs = slot_ptr<double>(c, S_XS), *ys = slot_ptr<double>(c, S_YS),
                 *vs = slot_ptr<double>(c, S_VS);
    const int2 *range = slot_ptr<int2>(c, S_RANGE);
    const int4 *cell = slot_ptr<int4>(c, S_CELL);
    TNode *tnode = slot_ptr<TNode>(c, S_TNODE);
    const Frame *frame = slot_ptr<Frame>(c, S_FRAME);
    if (order == ORDER_POTENTIAL)
        k_upward<ORDER_POTENTIAL><<<grid, UP_WARPS * 32, 0, c.stream>>>(
            nn, c.nsrc, c.leafcap, xs, ys, vs, range, cell, tnode, mass, w, wx, wy, exps, upcnt, frame,
            slot_ptr<unsigned>(c, S_ERR));
    else if (order == ORDER_FORCE)
        k_upward<ORDER_FORCE><<<grid, UP_WARPS * 32, 0, c.stream>>>(
            nn, c.nsrc, c.leafcap, xs, ys, vs, range, cell, tnode, mass, w, wx, wy, exps, upcnt, frame,
            slot_ptr<unsigned>(c, S_ERR));
    else {
        set_error(TC_ERR_INVALID, "unsupported expansion order %d", order);
        return TC_ERR_INVALID;
    }
    TC_KERNEL_CHECK();
    c.order = order;
    return TC_OK;
}

}  // namespace tc
