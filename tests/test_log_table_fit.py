"""The potential kernels' logarithm (log_pos in tc_math.cuh) on the CPU: its table and polynomial
are what fit_log_table.py writes, and the algorithm, restated here step by step with exact fused
multiply-adds, reproduces log x to within 2 ulp with the reduction index inside the table."""
import math
import os
import re
import struct
import sys
from fractions import Fraction

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "2d-treecodes_b200", "csrc")
HEADER = os.path.join(CSRC, "tc_log_table.cuh")


def header_values():
    src = open(HEADER).read()
    shift = int(re.search(r"LOG_KEY_SHIFT = (\d+);", src).group(1))
    base = int(re.search(r"LOG_IDX_BASE = (\d+);", src).group(1))
    ntab = int(re.search(r"LOG_NTAB = (\d+);", src).group(1))
    q = [float.fromhex(h) for h in re.findall(r"LOG_Q\d = (-?0x[0-9a-fp.+-]+);", src)]
    body = src[src.index("LOG_NEG_LOG_C[LOG_NTAB] = {"):]
    body = body[body.index("{") + 1:body.index("};")]
    table = [float.fromhex(h) for h in re.findall(r"-?0x[0-9a-f.]+p[+-]?\d+", body)]
    assert len(table) == ntab
    return shift, base, ntab, q, table


SHIFT, BASE, NTAB, Q, TABLE = header_values()
LN2 = float.fromhex("0x1.62e42fefa39efp-1")


def fma(a, b, c):
    """a * b + c with one rounding (exact rational arithmetic, then round to nearest)."""
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def words(x):
    u = struct.unpack("<Q", struct.pack("<d", x))[0]
    return u >> 32, u & 0xffffffff


def from_words(hi, lo):
    return struct.unpack("<d", struct.pack("<Q", ((hi & 0xffffffff) << 32) | lo))[0]


def f32_bits(f):
    return struct.unpack("<I", struct.pack("<f", f))[0]


def log_pos(x, rcp_ulps=0, trace=None):
    """log_pos step by step.  The reciprocal is the correctly rounded single-precision one moved
    by rcp_ulps units (the hardware's approximate reciprocal is within a few of it)."""
    hi, lo = words(x)
    ix = hi - 0x3fe6a09f
    e = ix >> 20                      # arithmetic shift (Python ints are signed)
    mf = ix & 0x000fffff
    m = from_words(mf + 0x3fe6a09f, lo)
    mfl = struct.unpack("<f", struct.pack("<I", (mf << 3) + (0x07e6a09f << 3)))[0]
    rc = f32_bits(float(np.float32(1.0) / np.float32(mfl))) + rcp_ulps
    key = (rc + (1 << (SHIFT - 1))) >> SHIFT
    c = from_words((key << (SHIFT - 3)) + (896 << 20), 0)
    r = fma(m, c, -1.0)
    idx = key - BASE
    if trace is not None:
        trace.append((idx, r, Fraction(m) * Fraction(c) - 1 == Fraction(r)))
    q = Q[-1]
    for j in reversed(range(len(Q) - 1)):
        q = fma(q, r, Q[j])
    p = fma(r * r, q, r)
    return fma(float(e), LN2, TABLE[idx] + p)


def test_log_table_regenerates():
    pytest.importorskip("mpmath")
    sys.path.insert(0, CSRC)
    try:
        import fit_log_table
    finally:
        sys.path.remove(CSRC)
    assert open(HEADER).read() == fit_log_table.header_text()


def arguments():
    r = np.random.default_rng(11)
    xs = list(np.exp(r.uniform(np.log(2e-15), np.log(1e6), 1500)))
    for b in [1.0, 2.0, 0.5, 2.0 ** -40, 2.0 ** 19, math.sqrt(2.0), math.sqrt(0.5)]:
        xs += [b, np.nextafter(b, 0), np.nextafter(b, 4 * b)]
        xs += list(b * (1 + np.linspace(-4e-3, 4e-3, 81)))
    # every reduction interval: m at both ends of each 10-bit reciprocal's range
    xs += list(np.linspace(math.sqrt(0.5), math.sqrt(2.0), 2400))
    xs += [float.fromhex("0x1.fffffffffffffp-1"), float.fromhex("0x1.0000000000001p+0"),
           float.fromhex("0x1.6a09e667f3bcdp+0"), float.fromhex("0x1.6a09effffffffp+0"),
           float.fromhex("0x1.6a09f00000000p+0"), float.fromhex("0x1p-1022"),
           float.fromhex("0x1.fffffffffffffp+1023")]
    return [float(x) for x in xs]


@pytest.mark.parametrize("rcp_ulps", [0, -6, 6])
def test_log_pos_reduction_is_exact_and_in_table(rcp_ulps):
    trace = []
    for x in arguments():
        log_pos(x, rcp_ulps, trace)
    idx = np.array([t[0] for t in trace])
    rmax = max(abs(t[1]) for t in trace)
    assert idx.min() >= 0 and idx.max() < NTAB, (idx.min(), idx.max())
    assert 20 <= idx.min() and idx.max() <= 532
    assert rmax <= 2.0 ** -10 * (1 + 2.0 ** -7), rmax
    assert all(t[2] for t in trace)   # r = m c - 1 exactly


def test_log_pos_within_two_ulp_of_the_exact_log():
    mp = pytest.importorskip("mpmath")
    worst = 0.0
    with mp.workdps(40):
        for x in arguments():
            got = log_pos(x)
            exact = mp.log(mp.mpf(x))
            ref = float(exact)
            ulp = math.ulp(abs(ref)) if ref != 0 else math.ulp(0.0)
            worst = max(worst, float(abs(mp.mpf(got) - exact)) / ulp)
    assert worst < 2.0, worst
