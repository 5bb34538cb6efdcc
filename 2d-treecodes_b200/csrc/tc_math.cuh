// tc_math.cuh -- binomial table and small complex helpers shared by the expansion kernels.
#pragma once

#include "tc_common.cuh"

namespace tc {

constexpr int BINOM_N = 2 * MAX_ORDER;

// Pascal's triangle in double (exact: every entry used, up to C(47,23) ~ 1.6e13, is below 2^53).
// The reference bakes the same integers into its kernels through kernels/binomial.py:1-5.
struct BinomTable {
    double c[BINOM_N][BINOM_N];
};

constexpr BinomTable make_binom_table() {
    BinomTable t{};
    for (int n = 0; n < BINOM_N; ++n) {
        t.c[n][0] = 1.0;
        for (int k = 1; k <= n; ++k) t.c[n][k] = t.c[n - 1][k - 1] + (k < n ? t.c[n - 1][k] : 0.0);
    }
    return t;
}

// Natural logarithm of a positive normal double, for the potential kernels' log r^2 terms
// (arguments r^2 + 10 eps or |z|^2 of a far cell, never zero, subnormal or infinite).  From the
// mathematics: x = 2^e m with m in [sqrt(1/2), sqrt(2)), s = (m - 1) / (m + 1), and
// log m = 2 atanh s = 2 s (1 + s^2 q(s^2)), q(z) = (atanh(sqrt z) / sqrt z - 1) / z; log x =
// e ln 2 + log m, with ln 2 split into a head of 21 bits (e * head exact) and a tail.  q is the
// degree-6 interpolant of it at the 7 first-kind Chebyshev nodes of z in [0, ((sqrt 2 - 1) /
// (sqrt 2 + 1))^2] (error below 2e-16, which the factor z <= 0.0295 scales to under 2^-57 of
// log m); fit_log_poly.py beside this file regenerates the coefficients.  The division is a refined reciprocal (rcp_nr).  About 25 instructions against the
// library log's ~100; within a few ulp of it (tests/test_gpu_parity.py checks the bound on
// 2^20 arguments).
__device__ __forceinline__ double log_pos(double x) {
    const int lo = __double2loint(x);
    int hi = __double2hiint(x);
    int e = (hi >> 20) - 1023;
    int mh = (hi & 0x000fffff) | 0x3ff00000;   // m in [1, 2)
    if (mh > 0x3ff6a09e) {                     // m above sqrt(2) (to 20 bits): halve it
        mh -= 0x00100000;
        ++e;
    }
    const double m = __hiloint2double(mh, lo);
    const double f = m - 1.0;
    const double s = f * rcp_nr(2.0 + f);
    const double z = s * s;
    double q = 0x1.2b584aae78a57p-4;
    q = fma(q, z, 0x1.39fe606542ddep-4);
    q = fma(q, z, 0x1.7462b4ab2ef6bp-4);
    q = fma(q, z, 0x1.c71c62e5800a1p-4);
    q = fma(q, z, 0x1.2492492df148dp-3);
    q = fma(q, z, 0x1.99999999952e2p-3);
    q = fma(q, z, 0x1.5555555555558p-2);
    const double two_s = 2.0 * s;
    const double logm = fma(two_s * z, q, two_s);
    constexpr double LN2_HEAD = 0x1.62e42p-1, LN2_TAIL = 0x1.fdf473de6af28p-22;
    const double de = (double)e;
    return fma(de, LN2_HEAD, fma(de, LN2_TAIL, logm));
}

struct cplx {
    double re, im;
};

__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

// a * b + c
__device__ __forceinline__ cplx cfma(cplx a, cplx b, cplx c) {
    return {fma(a.re, b.re, fma(-a.im, b.im, c.re)), fma(a.re, b.im, fma(a.im, b.re, c.im))};
}

// z^e for 0 <= e < 32 by square-and-multiply
__device__ __forceinline__ cplx cpow_int(cplx z, int e) {
    cplx r = {1.0, 0.0};
    cplx b = z;
#pragma unroll
    for (int bit = 0; bit < 5; ++bit) {
        if (e & (1 << bit)) r = cmul(r, b);
        b = cmul(b, b);
    }
    return r;
}

}  // namespace tc
