/*
 * oracle/kernel_probe.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Exported wrappers around the (hidden) restated ISPC kernels of ispc_kernels.cpp and
 * ispc_search.cpp, so that the CPU tests can check each kernel against the mathematics it
 * implements (kernels/*.m4, kernels/upward-common.ispc of the reference).
 */
typedef REAL realtype;

#include "upward-kernels.h"
#include "potential-kernels.h"
#include "force-kernels.h"

#define PROBE extern "C" __attribute__((visibility("default")))

PROBE int probe_order(void) { return ORDER; }

PROBE void probe_upward_setup(const double *x, const double *y, const double *v, int n,
                              double *out5)
{
    upward_setup(x, y, v, n, out5 + 0, out5 + 1, out5 + 2, out5 + 3, out5 + 4);
}

PROBE void probe_upward_p2e(const double *x, const double *y, const double *v, int n,
                            double xc, double yc, double *re, double *im)
{
    upward_p2e(x, y, v, n, xc, yc, re, im);
}

PROBE void probe_upward_e2e(const double *x0s, const double *y0s, const double *masses,
                            const double *exps /* 4 x 2 x ORDER */, double *re, double *im)
{
    const double *rx[4], *ix[4];
    for (int c = 0; c < 4; ++c) {
        rx[c] = exps + c * 2 * ORDER;
        ix[c] = exps + c * 2 * ORDER + ORDER;
    }
    upward_e2e(x0s, y0s, masses, rx, ix, re, im);
}

PROBE int probe_lower_bound(int s, int e, int val, const int *keys)
{
    return lower_bound_vec(s, e, val, keys);
}

PROBE int probe_upper_bound(int s, int e, int val, const int *keys)
{
    return upper_bound_vec(s, e, val, keys);
}

PROBE void probe_minmax(const double *x, const double *y, int n, double *out4)
{
    minmax_vec(x, y, n, out4);
}

#ifdef PROBE_POTENTIAL
PROBE double probe_potential_p2p(const double *x, const double *y, const double *v, int n,
                                 double xt, double yt)
{
    return potential_p2p(x, y, v, n, xt, yt);
}

PROBE double probe_potential_e2p(const double *rz, const double *iz, const double *m,
                                 const double *exps /* n x 2 x ORDER */, int n)
{
    const double *rx[16], *ix[16];
    for (int i = 0; i < n && i < 16; ++i) {
        rx[i] = exps + i * 2 * ORDER;
        ix[i] = exps + i * 2 * ORDER + ORDER;
    }
    return potential_e2p(rz, iz, m, rx, ix, n < 16 ? n : 16);
}
#else
PROBE void probe_force_p2p(const double *x, const double *y, const double *v, int n,
                           double x0, double y0, double h, double *xr, double *yr)
{
    force_p2p_8x8(x, y, v, n, x0, y0, h, xr, yr);
}

PROBE void probe_force_e2p(double m, double x0, double y0, double h, const double *exps,
                           double *xr, double *yr)
{
    force_e2p_8x8(m, x0, y0, h, exps, exps + ORDER, xr, yr);
}

PROBE void probe_e2l(const double *x0s, const double *y0s, const double *m,
                     const double *exps /* n x 2 x ORDER */, int n, double *rl, double *il)
{
    const double *rx[32], *ix[32];
    for (int i = 0; i < n && i < 32; ++i) {
        rx[i] = exps + i * 2 * ORDER;
        ix[i] = exps + i * 2 * ORDER + ORDER;
    }
    downward_e2l(x0s, y0s, m, rx, ix, n < 32 ? n : 32, rl, il);
}

PROBE void probe_l2p(double x0, double y0, double h, const double *rl, const double *il,
                     double *xr, double *yr)
{
    downward_l2p_8x8(x0, y0, h, rl, il, xr, yr);
}
#endif
