// tc_math.cuh -- binomial table and small complex helpers shared by the expansion kernels.
#pragma once

#include "tc_common.cuh"
#include "tc_log_table.cuh"

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
// (arguments r^2 + 10 eps or |z|^2 of a far cell, never zero, subnormal or infinite).
// Table-driven, after Tang's method (P. T. P. Tang, ACM TOMS 16(4), 1990): x = 2^e m with m in
// [sqrt(1/2), sqrt(2)); c = the single-precision reciprocal of m (from its top 20 fraction bits)
// rounded to 10 significant bits, so that r = m c - 1 is exact in one fma (m c has at most 62
// significant bits and |r| <= 2^-10 (1 + 2^-7)); log x = e ln 2 - log c + log1p(r), log1p(r) =
// r + r^2 q(r) with q of degree 3.  -log c comes from a table of LOG_NTAB doubles indexed by the
// rounded float bits of c, which the caller keeps in shared memory (load_log_table); m is in
// [sqrt(1/2), sqrt(2)) by construction, which puts the index in [20, 532] for any x.  The last
// step, e ln 2 + (-log c + log1p r), rounds twice: for e = 0 only the sum, and for e != 0 the
// result is at least ln 2 / 2 in size, so ln 2's own rounding (2^-55) stays below half an ulp of
// it.  fit_log_table.py beside this file writes the table and q (tc_log_table.cuh).  8 FP64
// operations, one single-precision reciprocal, one conversion and one shared load, against the
// library log's ~100 instructions; within 2 ulp of the exact logarithm (tests/test_gpu_parity.py
// checks 4 ulp against the library log on 2^20 arguments).
__device__ __forceinline__ double log_pos(double x, const double *__restrict__ neg_log_c) {
    const int ix = __double2hiint(x) - 0x3fe6a09f;   // high word of sqrt(1/2), rounded up
    const int e = ix >> 20;
    const int mf = ix & 0x000fffff;                 // fraction bits of m, offset
    const double m = __hiloint2double(mf + 0x3fe6a09f, __double2loint(x));
    const float mfl = __int_as_float((mf << 3) + (0x07e6a09f << 3));   // m to 20 bits, as float
    float rc;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rc) : "f"(mfl));
    // round the reciprocal to 10 significant bits: key = its float bits >> LOG_KEY_SHIFT
    const unsigned key = (__float_as_uint(rc) + (1u << (LOG_KEY_SHIFT - 1))) >> LOG_KEY_SHIFT;
    const double c = __hiloint2double((int)(key << (LOG_KEY_SHIFT - 3)) + (896 << 20), 0);
    const double r = fma(m, c, -1.0);
    double q = LOG_Q3;
    q = fma(q, r, LOG_Q2);
    q = fma(q, r, LOG_Q1);
    q = fma(q, r, LOG_Q0);
    const double p = fma(r * r, q, r);
    constexpr double LN2 = 0x1.62e42fefa39efp-1;
    return fma((double)e, LN2, neg_log_c[(int)key - LOG_IDX_BASE] + p);
}

// Copies log_pos's table into the block's shared memory; every thread of the block calls it.
__device__ __forceinline__ void load_log_table(double *s_neg_log_c) {
    for (int i = threadIdx.x; i < LOG_NTAB; i += blockDim.x) s_neg_log_c[i] = LOG_NEG_LOG_C[i];
    __syncthreads();
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
