#!/usr/bin/env python
"""Regenerates tc_log_table.cuh: the reduction table and the polynomial of log_pos (tc_math.cuh).

log_pos reduces x = 2^e m, m in [sqrt(1/2), sqrt(2)), with a short reciprocal c of m: c is the
single-precision reciprocal of m rounded to CBITS = 10 significant bits, so r = m c - 1 is exact
in one fma and |r| <= 2^-10 (1 + 2^-7) = R_MAX, and

    log x = e ln 2 - log c + log1p(r),   log1p(r) = r + r^2 q(r).

The table holds -log c, rounded to double, for every such c: entry i is the c whose float bits
are (IDX_BASE + i) << SHIFT (sign 0, 8 exponent bits, 9 fraction bits), covering c in
[0.6875, 1.4375), a margin around the [0.7070, 1.4142] that the reduction reaches.  q is the
degree-3 interpolant of (log1p(r) - r) / r^2 at the 4 first-kind Chebyshev nodes of [-R_MAX,
R_MAX] (its error, below 2^-47 of q, is scaled by r^2 / r <= 2^-10 in log1p).  Everything is
computed with 50 significant digits (mpmath) and rounded to the nearest double.

Run it to rewrite tc_log_table.cuh beside this file (`--check` compares instead).
"""
import os
import struct
import sys

import mpmath as mp

CBITS = 10                               # significant bits of c
SHIFT = 24 - CBITS                       # float bits of c >> SHIFT: the table key
IDX_BASE = 0x3f300000 >> SHIFT           # c = 0.6875
NTAB = (0x3fb80000 >> SHIFT) - IDX_BASE  # up to 1.4375 (exclusive)
DEGREE = 3
R_MAX = mp.mpf(2) ** -CBITS * (1 + mp.mpf(2) ** -7)
HEADER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tc_log_table.cuh")


def table_c(i):
    """The reciprocal c of table entry i (an exact float)."""
    return struct.unpack("<f", struct.pack("<I", (IDX_BASE + i) << SHIFT))[0]


def table(digits=50):
    """-log c_i rounded to double, i = 0 .. NTAB - 1."""
    with mp.workdps(digits):
        return [float(-mp.log(mp.mpf(table_c(i)))) for i in range(NTAB)]


def q_exact(r):
    """(log1p(r) - r) / r^2; its series -1/2 + r/3 - r^2/4 + ... next to 0 (the middle node)."""
    if abs(r) < mp.mpf(2) ** -40:
        return sum((-1) ** (k + 1) * r ** k / (k + 2) for k in range(8))
    return (mp.log1p(r) - r) / (r * r)


def coefficients(degree=DEGREE, digits=50):
    """Coefficients q_0..q_degree (double) of the interpolant, constant term first."""
    with mp.workdps(digits):
        n = degree + 1
        nodes = [R_MAX * mp.cos((2 * k + 1) * mp.pi / (2 * n)) for k in range(n)]
        a = mp.matrix(n, n)
        b = mp.matrix(n, 1)
        for i, r in enumerate(nodes):
            for j in range(n):
                a[i, j] = r ** j
            b[i] = q_exact(r)
        c = mp.lu_solve(a, b)
        return [float(c[j]) for j in range(n)]


def header_text():
    lines = [
        "// tc_log_table.cuh -- written by fit_log_table.py (do not edit): the reduction table and",
        "// the log1p polynomial of log_pos in tc_math.cuh.",
        "#pragma once",
        "",
        "namespace tc {",
        "",
        f"constexpr int LOG_KEY_SHIFT = {SHIFT};   // key = float bits of c >> LOG_KEY_SHIFT",
        f"constexpr int LOG_IDX_BASE = {IDX_BASE};   // key of entry 0",
        f"constexpr int LOG_NTAB = {NTAB};",
        "",
        f"// log1p(r) = r + r^2 q(r) on |r| <= 2^-{CBITS} (1 + 2^-7); q_0 .. q_{DEGREE}",
    ]
    for j, c in enumerate(coefficients()):
        lines.append(f"constexpr double LOG_Q{j} = {c.hex()};")
    lines += ["", "// -log c for c = float with bits (LOG_IDX_BASE + i) << LOG_KEY_SHIFT",
              "static __device__ const double LOG_NEG_LOG_C[LOG_NTAB] = {"]
    t = table()
    for i in range(0, NTAB, 3):
        lines.append("    " + " ".join(f"{v.hex()}," for v in t[i:i + 3]))
    lines += ["};", "", "}  // namespace tc", ""]
    return "\n".join(lines)


if __name__ == "__main__":
    text = header_text()
    if "--check" in sys.argv:
        ok = open(HEADER).read() == text
        print("tc_log_table.cuh is", "current" if ok else "STALE")
        sys.exit(0 if ok else 1)
    with open(HEADER, "w") as f:
        f.write(text)
    print("wrote", HEADER)
