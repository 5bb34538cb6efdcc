"""The coefficients of the potential kernels' logarithm (log_pos in tc_math.cuh) are the ones
its fitting script regenerates: the degree-6 Chebyshev interpolant of (atanh(sqrt z)/sqrt z -
1)/z on the reduced range, rounded to double."""
import os
import re
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "2d-treecodes_b200", "csrc")


def header_coefficients():
    """The seven q coefficients of log_pos, constant term first."""
    src = open(os.path.join(CSRC, "tc_math.cuh")).read()
    body = src[src.index("log_pos(double x)"):]
    body = body[:body.index("two_s")]
    lits = re.findall(r"(0x1\.[0-9a-f]+p-?\d+)", body)
    return [float.fromhex(h) for h in lits][::-1]


def test_log_poly_coefficients_regenerate():
    pytest.importorskip("mpmath")
    sys.path.insert(0, CSRC)
    try:
        import fit_log_poly
    finally:
        sys.path.remove(CSRC)
    got = header_coefficients()
    assert len(got) == 7
    assert fit_log_poly.coefficients() == got


def test_log_poly_accuracy_on_reduced_range():
    """The polynomial reproduces log m to well under a double ulp on the reduced range (checked
    in 50-digit arithmetic on 2001 points of m in [sqrt(1/2), sqrt(2)))."""
    mp = pytest.importorskip("mpmath")
    c = header_coefficients()
    with mp.workdps(50):
        lo, hi = mp.sqrt(mp.mpf(1) / 2), mp.sqrt(2)
        worst = mp.mpf(0)
        for i in range(2001):
            m = lo + (hi - lo) * i / 2001
            if m == 1:
                continue
            s = (m - 1) / (m + 1)
            z = s * s
            q = mp.mpf(0)
            for cj in reversed(c):
                q = q * z + mp.mpf(cj)
            approx = 2 * s * (1 + z * q)
            worst = max(worst, abs(approx - mp.log(m)) / abs(mp.log(m)))
        assert worst < 2.0 ** -56
