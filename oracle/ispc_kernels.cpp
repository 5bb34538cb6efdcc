/*
 * oracle/ispc_kernels.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A scalar C++ restatement of the twelve exported ISPC kernels of the reference
 * (kernels/upward-common.ispc, kernels/upward-kernels.m4, kernels/potential-kernels.m4,
 * kernels/force-kernels.m4).  The reference's ISPC/m4/bc toolchain is not available,
 * so these functions are linked against the reference's own C++ drivers (compiled
 * verbatim from drivers/*.cpp by oracle/Makefile) to form the CPU oracle.
 *
 * Prototypes come from the reference headers kernels/{upward,potential,force}-kernels.h,
 * which are included unchanged, so the symbols keep their names, signatures and
 * hidden visibility.
 *
 * The ISPC code runs a gang of programCount = 4 lanes (kernels/Makefile:28,
 * --target=avx2-i64x4).  The restatement keeps the per-lane accumulators of every
 * `foreach` (element i goes to lane i % 4) and reduces them with reduce4() below.
 *
 * Two compile-time modes:
 *   ORACLE_EXACT64      every constant and every log in double precision.
 *   (default) faithful  the m4-generated literals that carry no suffix are typed as
 *                       ISPC's default `float` (1/(n+1). in P2E, the bc "-1/l" prefactors,
 *                       the E2L binomials BINOMIAL(...).), and potential_p2p's main loop
 *                       takes a single-precision log, as written at
 *                       kernels/potential-kernels.m4:42.
 * Nothing under oracle/ is shipped or called by the product library.
 */
#include <cmath>
#include <cfloat>
#include <algorithm>

typedef REAL realtype;

#include "upward-kernels.h"
#include "potential-kernels.h"
#include "force-kernels.h"

namespace {

#ifdef ORACLE_EXACT64
typedef double lit_t;   /* unsuffixed m4 literals taken as double */
#else
typedef float lit_t;    /* unsuffixed m4 literals taken as ISPC float */
#endif

enum { LANES = 4 };

/* reduce_add over the 4 lanes of the gang: (l0 + l1) + (l2 + l3). */
inline double reduce4(const double v[LANES]) { return (v[0] + v[1]) + (v[2] + v[3]); }

/* Binomial coefficient C(n, k) as an exact integer (kernels/binomial.py:1-5). */
inline long long binomial(int n, int k)
{
    if (k < 0 || k > n) return 0;
    long long r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

/* Pairwise REDUCE macro of kernels/unroll.m4:42-48: combine neighbours
 * (a0+=a1, a2+=a3, ...), keep the even entries (plus an odd tail), repeat. */
inline double reduce_pairwise(double *a, int n)
{
    while (n > 1) {
        int m = 0;
        for (int i = 0; i < n; i += 2) {
            if (i + 1 < n) a[m++] = a[i] + a[i + 1];
            else a[m++] = a[i];
        }
        n = m;
    }
    return a[0];
}

} // namespace

/* ---------------------------------------------------------------------------
 * kernels/upward-common.ispc:13-57  upward_setup
 * msum/wsum/wxsum/wysum per lane, reduce_add; com per lane (note: a lane whose own
 * wsum is zero uses com = 0, because the ISPC condition tests the varying wsum);
 * radius = sqrt(max over lanes of max |x - com|^2).
 * ------------------------------------------------------------------------- */
extern "C" void upward_setup(const realtype xsources[], const realtype ysources[],
                             const realtype vsources[], const int nsources,
                             realtype * const mass, realtype * const weight,
                             realtype * const xsum, realtype * const ysum,
                             realtype * const radius)
{
    double msum[LANES] = {0, 0, 0, 0}, wsum[LANES] = {0, 0, 0, 0};
    double wxsum[LANES] = {0, 0, 0, 0}, wysum[LANES] = {0, 0, 0, 0};

    for (int i = 0; i < nsources; ++i) {
        const int l = i % LANES;
        const double x = xsources[i], y = ysources[i], m = vsources[i];
        const double w = std::fabs(m);
        msum[l] += m;
        wsum[l] += w;
        wxsum[l] += x * w;
        wysum[l] += y * w;
    }

    *mass = reduce4(msum);
    *weight = reduce4(wsum);
    *xsum = reduce4(wxsum);
    *ysum = reduce4(wysum);

    double xcom[LANES], ycom[LANES];
    for (int l = 0; l < LANES; ++l) {
        xcom[l] = wsum[l] != 0 ? *xsum / *weight : 0;
        ycom[l] = wsum[l] != 0 ? *ysum / *weight : 0;
    }

    double r2[LANES] = {0, 0, 0, 0};
    for (int i = 0; i < nsources; ++i) {
        const int l = i % LANES;
        const double xr = xsources[i] - xcom[l];
        const double yr = ysources[i] - ycom[l];
        r2[l] = std::max(r2[l], xr * xr + yr * yr);
    }

    *radius = std::sqrt(std::max(std::max(r2[0], r2[1]), std::max(r2[2], r2[3])));
}

/* ---------------------------------------------------------------------------
 * kernels/upward-common.ispc:126-150  minmax_vec (initial min 1e13, initial max 0)
 * ------------------------------------------------------------------------- */
extern "C" void minmax_vec(const realtype xsrc[], const realtype ysrc[], const int nsources,
                           realtype xmin_xmax_ymin_ymax[])
{
    const double big = (double)(lit_t)1e13;
    double lxmi = big, lymi = big, lxma = 0, lyma = 0;
    for (int i = 0; i < nsources; ++i) {
        lxmi = std::min(lxmi, xsrc[i]);
        lxma = std::max(lxma, xsrc[i]);
        lymi = std::min(lymi, ysrc[i]);
        lyma = std::max(lyma, ysrc[i]);
    }
    xmin_xmax_ymin_ymax[0] = lxmi;
    xmin_xmax_ymin_ymax[1] = lxma;
    xmin_xmax_ymin_ymax[2] = lymi;
    xmin_xmax_ymin_ymax[3] = lyma;
}

/* ---------------------------------------------------------------------------
 * kernels/upward-kernels.m4:18-93  upward_p2e (the active #else branch, :52-84)
 * a_n = -sum v (z - c)^(n+1) * (1/(n+1)),  n = 0..ORDER-1
 * ------------------------------------------------------------------------- */
extern "C" void upward_p2e(const realtype xsources[], const realtype ysources[],
                           const realtype vsources[], const int nsources,
                           const realtype xcom, const realtype ycom,
                           realtype * __restrict__ const rexpansions,
                           realtype * __restrict__ const iexpansions)
{
    double rxp[ORDER][LANES], ixp[ORDER][LANES];
    for (int n = 0; n < ORDER; ++n)
        for (int l = 0; l < LANES; ++l) rxp[n][l] = ixp[n][l] = 0;

    double invn[ORDER];
    for (int n = 0; n < ORDER; ++n) invn[n] = (double)((lit_t)1 / (lit_t)(n + 1));

    for (int i = 0; i < nsources; ++i) {
        const int l = i % LANES;
        const double rprod_0 = xsources[i] - xcom;
        const double iprod_0 = ysources[i] - ycom;
        const double src = vsources[i];

        double rtmp = rprod_0 * src;
        double itmp = iprod_0 * src;
        rxp[0][l] -= rtmp;
        ixp[0][l] -= itmp;

        double rprod = rprod_0, iprod = iprod_0;
        for (int n = 1; n < ORDER; ++n) {
            rtmp = rprod * rprod_0 - iprod * iprod_0;
            itmp = rprod * iprod_0 + iprod * rprod_0;
            const double term = src * invn[n];
            rprod = rtmp;
            iprod = itmp;
            rtmp = rprod * term;
            itmp = iprod * term;
            rxp[n][l] -= rtmp;
            ixp[n][l] -= itmp;
        }
    }

    for (int n = 0; n < ORDER; ++n) {
        rexpansions[n] = reduce4(rxp[n]);
        iexpansions[n] = reduce4(ixp[n]);
    }
}

/* ---------------------------------------------------------------------------
 * kernels/upward-kernels.m4:95-149  upward_e2e (one child per lane, 4 children)
 * b_l = z0^l [ -m/l + sum_{k=1..l} C(l-1,k-1) a_{k-1} z0^{-k} ],  l = 1..ORDER
 * z0^l is formed as conj(z0^-l) / |z0^-l|^2 (guarded against a zero modulus).
 * ------------------------------------------------------------------------- */
extern "C" void upward_e2e(const realtype x0s[], const realtype y0s[], const realtype masses[],
                           const realtype *vrxps[], const realtype *vixps[],
                           realtype rdstxp[], realtype idstxp[])
{
    double rinvz[LANES][ORDER + 1], iinvz[LANES][ORDER + 1];
    double rcoeff[LANES][ORDER + 1], icoeff[LANES][ORDER + 1];

    for (int c = 0; c < LANES; ++c) {
        const double x0 = x0s[c], y0 = y0s[c];
        const double r2z0 = x0 * x0 + y0 * y0;
        rinvz[c][1] = x0 / r2z0;
        iinvz[c][1] = -y0 / r2z0;
        for (int j = 2; j <= ORDER; ++j) {
            rinvz[c][j] = rinvz[c][j - 1] * rinvz[c][1] - iinvz[c][j - 1] * iinvz[c][1];
            iinvz[c][j] = rinvz[c][j - 1] * iinvz[c][1] + iinvz[c][j - 1] * rinvz[c][1];
        }
        for (int j = 1; j <= ORDER; ++j) {
            rcoeff[c][j] = vrxps[c][j - 1] * rinvz[c][j] - vixps[c][j - 1] * iinvz[c][j];
            icoeff[c][j] = vrxps[c][j - 1] * iinvz[c][j] + vixps[c][j - 1] * rinvz[c][j];
        }
    }

    for (int l = 1; l <= ORDER; ++l) {
        double rpart[LANES], ipart[LANES];
        for (int c = 0; c < LANES; ++c) {
            const double mass = masses[c];
            const double prefac = (l == 1) ? -mass : mass * (double)((lit_t)-1 / (lit_t)l);
            double rtmp = prefac;
            double itmp = 0;
            for (int k = 1; k <= l; ++k) {
                const double bin = (double)(float)binomial(l - 1, k - 1); /* ".f" literal */
                rtmp = rtmp + rcoeff[c][k] * bin;
                itmp = (k == 1) ? icoeff[c][k] * bin : itmp + icoeff[c][k] * bin;
            }
            const double invz2 = rinvz[c][l] * rinvz[c][l] + iinvz[c][l] * iinvz[c][l];
            const double invinvz2 = invz2 != 0 ? 1 / invz2 : 0;
            const double rz = rinvz[c][l] * invinvz2;
            const double iz = -iinvz[c][l] * invinvz2;
            rpart[c] = rtmp * rz - itmp * iz;
            ipart[c] = rtmp * iz + itmp * rz;
        }
        rdstxp[l - 1] = reduce4(rpart);
        idstxp[l - 1] = reduce4(ipart);
    }
}

/* ---------------------------------------------------------------------------
 * kernels/potential-kernels.m4:19-57  potential_p2p
 * 0.5 * sum v log(r^2 + 10 eps).  Main loop over groups of 16 with 4 accumulators
 * (lane l of accumulator j takes element i + l + 4 j); tail with a double log.
 * ------------------------------------------------------------------------- */
extern "C" realtype potential_p2p(const realtype * __restrict__ const _xsrc,
                                  const realtype * __restrict__ const _ysrc,
                                  const realtype * __restrict__ const _vsrc,
                                  const int nsources, const realtype xt, const realtype yt)
{
    const double eps = 10 * DBL_EPSILON;
    double s[4][LANES];
    for (int j = 0; j < 4; ++j)
        for (int l = 0; l < LANES; ++l) s[j][l] = 0;

    const int nnice = 16 * (nsources / 16);
    for (int i = 0; i < nnice; i += 16)
        for (int j = 0; j < 4; ++j)
            for (int l = 0; l < LANES; ++l) {
                const int k = i + l + 4 * j;
                const double xr = xt - _xsrc[k];
                const double yr = yt - _ysrc[k];
#ifdef ORACLE_EXACT64
                s[j][l] += std::log(xr * xr + yr * yr + eps) * _vsrc[k];
#else
                s[j][l] += (double)logf((float)(xr * xr + yr * yr + eps)) * _vsrc[k];
#endif
            }

    /* REDUCE(+=, s_0, s_1, s_2, s_3) */
    for (int l = 0; l < LANES; ++l) {
        s[0][l] += s[1][l];
        s[2][l] += s[3][l];
        s[0][l] += s[2][l];
    }

    for (int i = nnice; i < nsources; ++i) {
        const int l = (i - nnice) % LANES;
        const double xr = xt - _xsrc[i];
        const double yr = yt - _ysrc[i];
        s[0][l] += std::log(xr * xr + yr * yr + eps) * _vsrc[i];
    }

    return reduce4(s[0]) * 0.5;
}

/* ---------------------------------------------------------------------------
 * kernels/potential-kernels.m4:59-89  potential_e2p (one cell per lane)
 * sum over cells of m log(r^2)/2 + Re sum_{j=1..p} a_{j-1} z^{-j}
 * ------------------------------------------------------------------------- */
extern "C" realtype potential_e2p(const realtype *rzs, const realtype *izs, const realtype *masses,
                                  const realtype * const *rxps, const realtype * const *ixps,
                                  const int ndst)
{
    double result[LANES] = {0, 0, 0, 0};
    for (int i = 0; i < ndst; ++i) {
        const int l = i % LANES;
        const double rz = rzs[i], iz = izs[i];
        const double r2 = rz * rz + iz * iz;
        double rinvz[ORDER + 1], iinvz[ORDER + 1];
        rinvz[1] = rz / r2;
        iinvz[1] = -iz / r2;
        for (int j = 2; j <= ORDER; ++j) {
            rinvz[j] = rinvz[j - 1] * rinvz[1] - iinvz[j - 1] * iinvz[1];
            iinvz[j] = rinvz[j - 1] * iinvz[1] + iinvz[j - 1] * rinvz[1];
        }
        double rsum[ORDER];
        for (int j = 1; j <= ORDER; ++j)
            rsum[j - 1] = rxps[i][j - 1] * rinvz[j] - ixps[i][j - 1] * iinvz[j];
        const double series = reduce_pairwise(rsum, ORDER);
        result[l] += masses[i] * std::log(r2) / 2 + series;
    }
    return reduce4(result);
}

/* ---------------------------------------------------------------------------
 * kernels/force-kernels.m4:15-55  force_p2p_8x8
 * result[ix + 8 iy] += v (xr, yr) / (xr^2 + (yr^2 + 10 eps)),  target (x0 + ix h, y0 + iy h)
 * ------------------------------------------------------------------------- */
extern "C" void force_p2p_8x8(const realtype * __restrict__ const xsources,
                              const realtype * __restrict__ const ysources,
                              const realtype * __restrict__ const vsources,
                              const int nsources, const realtype x0, const realtype y0,
                              const realtype h, realtype * const xresult, realtype * const yresult)
{
    const double eps = 10 * DBL_EPSILON;
    double xt[8], yt[8];
    for (int ix = 0; ix < 8; ++ix) xt[ix] = x0 + ix * h;
    for (int iy = 0; iy < 8; ++iy) yt[iy] = y0 + iy * h;

    for (int s = 0; s < nsources; ++s) {
        const double xsrc = xsources[s], ysrc = ysources[s], vsrc = vsources[s];
        double xr[8], xr2[8], yr[8], yr2[8];
        for (int ix = 0; ix < 8; ++ix) {
            xr[ix] = xt[ix] - xsrc;
            xr2[ix] = xr[ix] * xr[ix];
        }
        for (int iy = 0; iy < 8; ++iy) {
            yr[iy] = yt[iy] - ysrc;
            yr2[iy] = yr[iy] * yr[iy] + eps;
        }
        for (int iy = 0; iy < 8; ++iy)
            for (int ix = 0; ix < 8; ++ix) {
                const double factor = vsrc / (xr2[ix] + yr2[iy]);
                xresult[ix + 8 * iy] += xr[ix] * factor;
                yresult[ix + 8 * iy] += yr[iy] * factor;
            }
    }
}

/* ---------------------------------------------------------------------------
 * kernels/force-kernels.m4:57-98  force_e2p_8x8
 * w = m/z - sum_{j=0..p-1} (j+1) a_j z^{-(j+2)};  x += Re w, y -= Im w
 * ------------------------------------------------------------------------- */
extern "C" void force_e2p_8x8(const realtype mass, const realtype x0, const realtype y0,
                              const realtype h, const realtype * __restrict__ const rxp,
                              const realtype * __restrict__ const ixp,
                              realtype * const xresult, realtype * const yresult)
{
    for (int d = 0; d < 64; ++d) {
        const int ix = d & 7, iy = d >> 3;
        const double rz = x0 + ix * h;
        const double iz = y0 + iy * h;
        const double r2 = rz * rz + iz * iz;
        const double rinvz_1 = rz / r2;
        const double iinvz_1 = -iz / r2;
        double rsum = mass * rinvz_1, isum = mass * iinvz_1;
        double rprod = rinvz_1, iprod = iinvz_1;
        for (int j = 0; j < ORDER; ++j) {
            const double rtmp = rprod * rinvz_1 - iprod * iinvz_1;
            const double itmp = rprod * iinvz_1 + iprod * rinvz_1;
            rprod = rtmp;
            iprod = itmp;
            rsum -= (j + 1) * (rxp[j] * rprod - ixp[j] * iprod);
            isum -= (j + 1) * (rxp[j] * iprod + ixp[j] * rprod);
        }
        xresult[d] += rsum;
        yresult[d] -= isum;
    }
}

/* ---------------------------------------------------------------------------
 * kernels/force-kernels.m4:102-155  downward_e2l (cells in groups of 4 lanes)
 * L_l += z0^{-l} [ -m/l + sum_{k=1..p} (-1)^k C(l+k-1,k-1) a_{k-1} z0^{-k} ],  l = 1..p
 * ------------------------------------------------------------------------- */
extern "C" void downward_e2l(const realtype *x0s, const realtype *y0s, const realtype *masses,
                             const realtype * __restrict__ * const vrexpansions,
                             const realtype * __restrict__ * const viexpansions,
                             const int nexpansions, realtype * __restrict__ const rlocal,
                             realtype * __restrict__ const ilocal)
{
    static double bin[ORDER + 1][ORDER + 1];
    static bool init = false;
    if (!init) {
        for (int l = 1; l <= ORDER; ++l)
            for (int k = 1; k <= ORDER; ++k)
                bin[l][k] = (double)(lit_t)binomial(l + k - 1, k - 1);
        init = true;
    }

    for (int g = 0; g < nexpansions; g += LANES) {
        double rpart[ORDER + 1][LANES], ipart[ORDER + 1][LANES];
        for (int l = 0; l <= ORDER; ++l)
            for (int c = 0; c < LANES; ++c) rpart[l][c] = ipart[l][c] = 0;

        for (int c = 0; c < LANES && g + c < nexpansions; ++c) {
            const int i = g + c;
            const double mass = masses[i], x0 = x0s[i], y0 = y0s[i];
            const double r2z0 = x0 * x0 + y0 * y0;
            double rinvz[ORDER + 1], iinvz[ORDER + 1], rcoeff[ORDER + 1], icoeff[ORDER + 1];
            rinvz[1] = x0 / r2z0;
            iinvz[1] = -y0 / r2z0;
            for (int j = 2; j <= ORDER; ++j) {
                rinvz[j] = rinvz[j - 1] * rinvz[1] - iinvz[j - 1] * iinvz[1];
                iinvz[j] = rinvz[j - 1] * iinvz[1] + iinvz[j - 1] * rinvz[1];
            }
            const realtype *rxp = vrexpansions[i], *ixp = viexpansions[i];
            for (int j = 1; j <= ORDER; ++j) {
                rcoeff[j] = rxp[j - 1] * rinvz[j] - ixp[j - 1] * iinvz[j];
                icoeff[j] = rxp[j - 1] * iinvz[j] + ixp[j - 1] * rinvz[j];
            }
            for (int l = 1; l <= ORDER; ++l) {
                double rtmp = (l == 1) ? -mass : mass * (double)((lit_t)-1 / (lit_t)l);
                double itmp = 0;
                for (int k = 1; k <= ORDER; ++k) {
                    if (k & 1) {
                        rtmp -= bin[l][k] * rcoeff[k];
                        itmp -= bin[l][k] * icoeff[k];
                    } else {
                        rtmp += bin[l][k] * rcoeff[k];
                        itmp += bin[l][k] * icoeff[k];
                    }
                }
                rpart[l][c] = rtmp * rinvz[l] - itmp * iinvz[l];
                ipart[l][c] = rtmp * iinvz[l] + itmp * rinvz[l];
            }
        }
        for (int l = 1; l <= ORDER; ++l) {
            rlocal[l] += reduce4(rpart[l]);
            ilocal[l] += reduce4(ipart[l]);
        }
    }
}

/* ---------------------------------------------------------------------------
 * kernels/force-kernels.m4:157-191  downward_l2p_8x8
 * sum_{l=1..p} l L_l z^{l-1}, z = (x0 + ix h, y0 + iy h);  x += Re, y -= Im
 * ------------------------------------------------------------------------- */
extern "C" void downward_l2p_8x8(const realtype x0, const realtype y0, const realtype h,
                                 const realtype * __restrict__ const rlocal,
                                 const realtype * __restrict__ const ilocal,
                                 realtype * const xresult, realtype * const yresult)
{
    for (int d = 0; d < 64; ++d) {
        const int ix = d & 7, iy = d >> 3;
        const double rz_1 = x0 + ix * h;
        const double iz_1 = y0 + iy * h;
        double rres = rlocal[1], ires = ilocal[1];
        double rz = rz_1, iz = iz_1; /* z^(l-1) */
        for (int l = 2; l <= ORDER; ++l) {
            rres = rres + l * (rlocal[l] * rz - ilocal[l] * iz);
            ires = ires + l * (rlocal[l] * iz + ilocal[l] * rz);
            const double rzn = rz * rz_1 - iz * iz_1;
            const double izn = rz * iz_1 + iz * rz_1;
            rz = rzn;
            iz = izn;
        }
        xresult[d] += rres;
        yresult[d] -= ires;
    }
}
