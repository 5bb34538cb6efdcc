// upward.cu -- the upward pass: leaf setup + P2E, then E2E level by level.
//
// k_upward_leaves: persistent warps, one leaf at a time (drivers/upward.cpp:61-93,
// kernels/upward-common.ispc:13-57, kernels/upward-kernels.m4:18-93).
// k_upward_level: one launch per tree level, deepest first; one warp per inner node merges its
// four children and shifts their expansions into it (upward.cpp:95-218,
// kernels/upward-kernels.m4:95-149).  Children were finished by the previous launch, so no
// atomics or fences are needed; the reference does the same merges in the order its OpenMP
// tasks happen to finish.
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
#include <algorithm>

#include "tc_internal.h"
#include "tc_math.cuh"

namespace tc {

__constant__ BinomTable c_binom_up = make_binom_table();

constexpr int UP_WARPS = 4;
constexpr int UP_CHUNK = 256;   // leaf sources staged in shared memory per pass (multiple of 4)

// Per-warp scratch of the leaf kernel; the phases of a leaf use it one after the other.
template <int P>
struct LeafShared {
    union {
        struct {
            double sx[UP_CHUNK], sy[UP_CHUNK], sv[UP_CHUNK];   // staged leaf sources (setup)
        } stage;
        struct {
            double re[32][P + 1], im[32][P + 1];   // v z^(n+1) of a 32-source chunk (P2E)
        } terms;
    };
};

// Per-warp scratch of the merge kernel.
template <int P>
struct MergeShared {
    double zr[4][P + 1], zi[4][P + 1];   // z0^-k per child
    double cr[4][P + 1], ci[4][P + 1];   // a_{k-1} z0^-k per child
    double pr[4][P], pi[4][P];           // shifted contribution of child c to coefficient l
};

__device__ __forceinline__ bool is_leaf(int2 rg, int4 cl, int leafcap) {
    return (rg.y - rg.x <= leafcap) || cl.x == LMAX;
}

// ------------------------------------------------------------------------------ leaves
template <int P>
__device__ __forceinline__ void upward_leaf(
    int node, int nnodes, int nsrc, int leafcap, const double *__restrict__ xs,
    const double *__restrict__ ys, const double *__restrict__ vs, const int2 *__restrict__ range,
    const int4 *__restrict__ cell, TNode *tnode, double *mass, double *wgt, double *wxs,
    double *wys, double *exps, const Frame *__restrict__ frame, unsigned *err,
    LeafShared<P> &sh) {
    const int lane = lane_id();
    const int2 rg = range[node];
    const int4 cl = cell[node];
    if (!is_leaf(rg, cl, leafcap)) return;
    if (rg.x < 0 || rg.y < rg.x || rg.y > nsrc || cl.w >= nnodes || cl.x < 0 || cl.x > LMAX) {
        if (lane == 0) atomicOr(err, DEVERR_BOUNDS);
        return;
    }
    const Frame f = *frame;
    const int s = rg.x, e = rg.y;

    // Leaf sources pass through shared memory in chunks of UP_CHUNK (coalesced loads by all
    // lanes); a leaf that fits one chunk is loaded once for both setup passes.
    const int nch = (e - s + UP_CHUNK - 1) / UP_CHUNK;
    auto stage = [&](int c0, int cnt) {
        __syncwarp();
        for (int j = lane; j < cnt; j += 32) {
            sh.stage.sx[j] = xs[c0 + j];
            sh.stage.sy[j] = ys[c0 + j];
            sh.stage.sv[j] = vs[c0 + j];
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
#pragma unroll 4
            for (int j = lane; j < cnt; j += 4) {
                const double x = sh.stage.sx[j], y = sh.stage.sy[j], m = sh.stage.sv[j];
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
#pragma unroll 4
                for (int j = lane; j < cnt; j += 4) {
                    const double xr = __dsub_rn(sh.stage.sx[j], lx), yr = __dsub_rn(sh.stage.sy[j], ly);
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

    // ---- upward_p2e: a_n = -sum v (z - c)^(n+1) / (n+1).  For each chunk of 32 sources, lane i
    // writes the terms v z_i^(n+1) of its source to shared memory (row i); lane n then adds up
    // column n.  No per-lane coefficient arrays and no cross-lane reduction are needed.
    double accr = 0, acci = 0;
    for (int c0 = s; c0 < e; c0 += 32) {
        const int cnt = min(32, e - c0);
        __syncwarp();
        if (lane < cnt) {
            const double r0 = xs[c0 + lane] - xcom, i0 = ys[c0 + lane] - ycom;
            const double v = vs[c0 + lane];
            double pr = r0, pim = i0;
#pragma unroll
            for (int n = 0; n < P; ++n) {
                sh.terms.re[lane][n] = pr * v;
                sh.terms.im[lane][n] = pim * v;
                const double tr = pr * r0 - pim * i0;
                const double ti = pr * i0 + pim * r0;
                pr = tr;
                pim = ti;
            }
        }
        __syncwarp();
        if (lane < P)
            for (int i = 0; i < cnt; ++i) {
                accr += sh.terms.re[i][lane];
                acci += sh.terms.im[i][lane];
            }
    }
    __syncwarp();
    double *ex = exps + (size_t)node * 2 * P;
    if (lane < P) {
        const double f = -1.0 / (lane + 1);
        ex[lane] = accr * f;
        ex[P + lane] = acci * f;
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

}

template <int P>
__global__ __launch_bounds__(UP_WARPS * 32) void k_upward_leaves(
    int nnodes, int nsrc, int leafcap, const double *__restrict__ xs, const double *__restrict__ ys,
    const double *__restrict__ vs, const int2 *__restrict__ range, const int4 *__restrict__ cell,
    TNode *tnode, double *mass, double *wgt, double *wxs, double *wys, double *exps,
    const Frame *__restrict__ frame, unsigned *err) {
    extern __shared__ __align__(16) unsigned char leaf_smem[];
    LeafShared<P> *shared = reinterpret_cast<LeafShared<P> *>(leaf_smem);
    const int warp = threadIdx.x >> 5;
    for (int node = blockIdx.x * UP_WARPS + warp; node < nnodes; node += gridDim.x * UP_WARPS)
        upward_leaf<P>(node, nnodes, nsrc, leafcap, xs, ys, vs, range, cell, tnode, mass, wgt,
                       wxs, wys, exps, frame, err, shared[warp]);
}

// ------------------------------------------------------------------------------ merge (E2E)
// b_l = sum_c z0^l [ -m/l + sum_{k=1..l} C(l-1,k-1) a_{k-1} z0^-k ], z0 = child com - parent com
template <int P>
__device__ void shift_children(MergeShared<P> &sh, const double *exps, int cb, const double *cm,
                               const double *cx, const double *cy, double px, double py,
                               double *dst, const double (*bin)[P]) {
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
        const double ar = ex[k - 1], ai = ex[P + k - 1];
        sh.cr[c][k] = ar * sh.zr[c][k] - ai * sh.zi[c][k];
        sh.ci[c][k] = ar * sh.zi[c][k] + ai * sh.zr[c][k];
    }
    __syncwarp();
    // P lanes; lane j takes children (0,1) or (2,3) and the coefficient pair (l, P + 1 - l), so
    // every busy lane runs the same 2 * (P + 1) inner iterations.
    if (lane < P) {
        const int half = P / 2;
        const int c0 = lane < half ? 0 : 2;
        const int jj = lane % half;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int l = q == 0 ? jj + 1 : P - jj;
            const double minv = -1.0 / l;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int c = c0 + cc;
                double rtmp = l == 1 ? -cm[c] : cm[c] * minv;
                double itmp = 0;
                for (int k = 1; k <= l; ++k) {
                    const double b = bin[k - 1][l - 1];
                    rtmp += sh.cr[c][k] * b;
                    itmp += sh.ci[c][k] * b;
                }
                const double zr = sh.zr[c][l], zi = sh.zi[c][l];
                const double invz2 = zr * zr + zi * zi;
                const double inv = invz2 != 0 ? 1.0 / invz2 : 0.0;
                const double rz = zr * inv, iz = -zi * inv;
                sh.pr[c][l - 1] = rtmp * rz - itmp * iz;
                sh.pi[c][l - 1] = rtmp * iz + itmp * rz;
            }
        }
    }
    __syncwarp();
    if (lane < P) {
        dst[lane] = (sh.pr[0][lane] + sh.pr[1][lane]) + (sh.pr[2][lane] + sh.pr[3][lane]);
        dst[P + lane] = (sh.pi[0][lane] + sh.pi[1][lane]) + (sh.pi[2][lane] + sh.pi[3][lane]);
    }
    __syncwarp();
}

template <int P>
__global__ __launch_bounds__(UP_WARPS * 32) void k_upward_level(
    int lo, int hi, int nnodes, int leafcap, const int2 *__restrict__ range,
    const int4 *__restrict__ cell, TNode *tnode, double *mass, double *wgt, double *wxs,
    double *wys, double *exps, const Frame *__restrict__ frame, unsigned *err) {
    __shared__ MergeShared<P> shared[UP_WARPS];
    __shared__ double s_bin[P][P];   // s_bin[k-1][l-1] = C(l-1, k-1): lane l reads a row
    for (int i = threadIdx.x; i < P * P; i += blockDim.x) {
        const int k = i / P, l = i % P;
        s_bin[k][l] = c_binom_up.c[l][k];
    }
    __syncthreads();
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    MergeShared<P> &sh = shared[warp];
    const double ext = frame->ext;
    for (int parent = lo + blockIdx.x * UP_WARPS + warp; parent < hi;
         parent += gridDim.x * UP_WARPS) {
        const int2 prg = range[parent];
        const int4 pcl = cell[parent];
        if (is_leaf(prg, pcl, leafcap)) continue;
        const int cb = tnode[parent].child;
        if (cb <= parent || cb + 4 > nnodes) {
            if (lane == 0) atomicOr(err, DEVERR_BOUNDS);
            continue;
        }
        double cm[4], cw[4], cwx[4], cwy[4], cxc[4], cyc[4], cr[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            cm[c] = mass[cb + c];
            cw[c] = wgt[cb + c];
            cwx[c] = wxs[cb + c];
            cwy[c] = wys[cb + c];
            cxc[c] = tnode[cb + c].xcom;
            cyc[c] = tnode[cb + c].ycom;
            cr[c] = tnode[cb + c].r;
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
        const double cap = __ddiv_rn(__dmul_rn((double)1.4143f, ext), (double)(1 << pcl.x));
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
            for (int k = lane; k < 2 * P; k += 32) dst[k] = src[k];
        } else {
            shift_children<P>(sh, exps, cb, cm, cxc, cyc, px, py, dst, s_bin);
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
        __syncwarp();
    }
}

static int sm_count_up() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

template <int P>
static int run_upward(Context &c, double *mass, double *w, double *wx, double *wy, double *exps) {
    const int nn = c.nnodes;
    const double *xs = slot_ptr<double>(c, S_XS), *ys = slot_ptr<double>(c, S_YS),
                 *vs = slot_ptr<double>(c, S_VS);
    const int2 *range = slot_ptr<int2>(c, S_RANGE);
    const int4 *cell = slot_ptr<int4>(c, S_CELL);
    TNode *tnode = slot_ptr<TNode>(c, S_TNODE);
    const Frame *frame = slot_ptr<Frame>(c, S_FRAME);
    unsigned *err = slot_ptr<unsigned>(c, S_ERR);
    const int sms = sm_count_up();

    static int occ = 0;
    const size_t smem = UP_WARPS * sizeof(LeafShared<P>);
    if (!occ) {
        TC_CUDA_TRY(cudaFuncSetAttribute(k_upward_leaves<P>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        TC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_upward_leaves<P>,
                                                                  UP_WARPS * 32, smem));
        occ = std::max(occ, 1);
    }
    const int grid = (int)std::min<long long>((nn + UP_WARPS - 1) / UP_WARPS, (long long)sms * occ);
    k_upward_leaves<P><<<grid, UP_WARPS * 32, smem, c.stream>>>(
        nn, c.nsrc, c.leafcap, xs, ys, vs, range, cell, tnode, mass, w, wx, wy, exps, frame, err);
    TC_KERNEL_CHECK();
    // inner nodes exist on levels 0 .. LMAX-1; level l occupies [level_off[l], level_off[l+1])
    for (int l = LMAX - 1; l >= 0; --l) {
        const int lo = c.level_off[l], hi = c.level_off[l + 1];
        if (hi <= lo) continue;
        const int g = (int)std::min<long long>((hi - lo + UP_WARPS - 1) / UP_WARPS, (long long)sms * 8);
        k_upward_level<P><<<g, UP_WARPS * 32, 0, c.stream>>>(lo, hi, nn, c.leafcap, range, cell,
                                                             tnode, mass, w, wx, wy, exps, frame, err);
        TC_KERNEL_CHECK();
    }
    return TC_OK;
}

int upward_pass(Context &c, int order) {
    const int nn = c.nnodes;
    int rc;
    double *mass, *w, *wx, *wy, *exps;
    if ((rc = ensure(c, S_MASS, nn, &mass)) || (rc = ensure(c, S_W, nn, &w)) ||
        (rc = ensure(c, S_WX, nn, &wx)) || (rc = ensure(c, S_WY, nn, &wy)) ||
        (rc = ensure(c, S_EXPS, (size_t)nn * 2 * order, &exps)))
        return rc;
    if (order == ORDER_POTENTIAL)
        rc = run_upward<ORDER_POTENTIAL>(c, mass, w, wx, wy, exps);
    else if (order == ORDER_FORCE)
        rc = run_upward<ORDER_FORCE>(c, mass, w, wx, wy, exps);
    else {
        set_error(TC_ERR_INVALID, "unsupported expansion order %d", order);
        return TC_ERR_INVALID;
    }
    if (rc) return rc;
    c.order = order;
    return TC_OK;
}

}  // namespace tc
