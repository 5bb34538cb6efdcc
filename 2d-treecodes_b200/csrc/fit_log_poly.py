#!/usr/bin/env python
"""Regenerates the seven coefficients of q(z) in log_pos (tc_math.cuh).

log m = 2 atanh(s) = 2 s (1 + s^2 q(s^2)) for s = (m - 1) / (m + 1), m in [sqrt(1/2), sqrt(2)),
with q(z) = (atanh(sqrt z) / sqrt z - 1) / z = 1/3 + z/5 + z^2/7 + ...  The polynomial is the
degree-6 interpolant of q at the 7 Chebyshev nodes of the first kind on [0, zmax], zmax =
((sqrt 2 - 1) / (sqrt 2 + 1))^2, computed with 50 significant digits (mpmath) and rounded to
double.  Run it to print the coefficients, constant term first, as C hex literals.
"""
import mpmath as mp

DEGREE = 6


def coefficients(degree=DEGREE, digits=50):
    """Coefficients c_0..c_degree (double) of the interpolant, constant term first."""
    with mp.workdps(digits):
        s2 = mp.sqrt(2)
        zmax = ((s2 - 1) / (s2 + 1)) ** 2
        n = degree + 1
        nodes = [zmax / 2 * (1 - mp.cos((2 * k + 1) * mp.pi / (2 * n))) for k in range(n)]

        def q(z):
            r = mp.sqrt(z)
            return (mp.atanh(r) / r - 1) / z

        a = mp.matrix(n, n)
        b = mp.matrix(n, 1)
        for i, z in enumerate(nodes):
            for j in range(n):
                a[i, j] = z ** j
            b[i] = q(z)
        c = mp.lu_solve(a, b)
        return [float(c[j]) for j in range(n)]


if __name__ == "__main__":
    for j, c in enumerate(coefficients()):
        print(f"c{j} = {c.hex()}")
