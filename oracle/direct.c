/*
 * oracle/direct.c -- TEST INFRASTRUCTURE ONLY (the accuracy oracle).
 *
 * The O(N M) FP64 direct sums with which the reference verifies itself
 * (main.cpp:201-245), evaluated on a caller-chosen subset of targets:
 *   potential: sum_j v_j log(sqrt(r^2 + eps))            (main.cpp:213-221)
 *   force:     sum_j v_j (xr, yr) / (r^2 + eps)          (main.cpp:232-243)
 * with eps = 10 * DBL_EPSILON (main.cpp:175).
 * Also the reference's pass rule check() (main.cpp:31-58).
 */
#include <float.h>
#include <math.h>

void oracle_direct_potential(const double *xs, const double *ys, const double *vs, int n,
                             const double *xt, const double *yt, int m, double *out)
{
    const double eps = DBL_EPSILON * 10;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < m; ++i) {
        const double xd = xt[i], yd = yt[i];
        double s = 0;
        for (int j = 0; j < n; ++j) {
            const double xr = xd - xs[j];
            const double yr = yd - ys[j];
            const double r = sqrt(xr * xr + yr * yr + eps);
            s += log(r) * vs[j];
        }
        out[i] = s;
    }
}

void oracle_direct_force(const double *xs, const double *ys, const double *vs, int n,
                         const double *xt, const double *yt, int m, double *xout, double *yout)
{
    const double eps = DBL_EPSILON * 10;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < m; ++i) {
        const double xd = xt[i], yd = yt[i];
        double sx = 0, sy = 0;
        for (int j = 0; j < n; ++j) {
            const double xr = xd - xs[j];
            const double yr = yd - ys[j];
            const double factor = vs[j] / (xr * xr + yr * yr + eps);
            sx += xr * factor;
            sy += yr * factor;
        }
        xout[i] = sx;
        yout[i] = sy;
    }
}

/* main.cpp:31-58: returns 1 when every point passes |rel| < tol || |abs| < tol,
 * with rel = err / max(1e-6, max(|res|, |ref|)); stats = {linf, l1, linf_rel, l1_rel}. */
int oracle_check(const double *ref, const double *res, int n, double tol, double *stats)
{
    double linf = 0, l1 = 0, linf_rel = 0, l1_rel = 0;
    int ok = 1;
    for (int i = 0; i < n; ++i) {
        if (isnan(ref[i]) || isnan(res[i])) { ok = 0; continue; }
        const double err = ref[i] - res[i];
        const double maxval = fmax(fabs(res[i]), fabs(ref[i]));
        const double relerr = err / fmax(1e-6, maxval);
        if (!(fabs(relerr) < tol || fabs(err) < tol)) ok = 0;
        l1 += fabs(err);
        l1_rel += fabs(relerr);
        linf = fmax(linf, fabs(err));
        linf_rel = fmax(linf_rel, fabs(relerr));
    }
    stats[0] = linf;
    stats[1] = l1;
    stats[2] = linf_rel;
    stats[3] = l1_rel;
    return ok;
}
