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
