"""CPU checks of the oracle: the restated ISPC kernels against the mathematics they implement,
the reference's own verifier (direct sum, main.cpp:31-58 pass rule) on the full oracle, the
k-ary searches against exact bounds, and the golden fixtures reproduced bit for bit."""
import ctypes
import glob
import os

import numpy as np
import pytest

import oracle as O
import workloads as W

pytestmark = pytest.mark.skipif(not O.available(), reason="oracle libraries not built")

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def probe(kind, mode="exact64"):
    L = ctypes.CDLL(os.path.join(O.REF_DIR, f"libprobe_{kind}_{mode}.so"))
    if kind == "potential":
        L.probe_potential_p2p.restype = ctypes.c_double
        L.probe_potential_p2p.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.probe_potential_e2p.restype = ctypes.c_double
        L.probe_potential_e2p.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int]
    else:
        L.probe_force_p2p.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, _dp, _dp]
        L.probe_force_e2p.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, _dp, _dp, _dp]
        L.probe_e2l.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, _dp, _dp]
        L.probe_l2p.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp]
    L.probe_upward_p2e.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp]
    L.probe_upward_e2e.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp]
    L.probe_upward_setup.argtypes = [_dp, _dp, _dp, ctypes.c_int, _dp]
    L.probe_lower_bound.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip]
    L.probe_upper_bound.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip]
    L.probe_order.restype = ctypes.c_int
    return L


def P(a):
    return a.ctypes.data_as(_dp)


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.mark.parametrize("kind", ["potential", "force"])
def test_kary_search_matches_exact_bounds(kind):
    """kernels/upward-common.ispc:59-124 restated: the 4-lane k-ary searches return the exact
    lower/upper bound (the child boundaries of upward.cpp:264-265)."""
    L = probe(kind)
    r = np.random.default_rng(3)
    for trial in range(300):
        n = int(r.integers(1, 5000))
        keys = np.sort(r.integers(0, 1 << int(r.integers(2, 31)), n)).astype(np.int32)
        kp = keys.ctypes.data_as(_ip)
        for _ in range(20):
            s = int(r.integers(0, n))
            e = int(r.integers(s + 1, n + 1))
            val = int(keys[r.integers(s, e)]) + int(r.integers(-2, 3))
            lo = s + int(np.searchsorted(keys[s:e], val, "left"))
            hi = s + int(np.searchsorted(keys[s:e], val, "right"))
            assert L.probe_lower_bound(s, e, val, kp) == lo
            assert L.probe_upper_bound(s, e, val, kp) == hi


@pytest.mark.parametrize("kind", ["potential", "force"])
def test_p2e_matches_multipole_formula(kind):
    """upward-kernels.m4:18-93: a_k = -sum v (z - c)^(k+1) / (k+1)."""
    L = probe(kind)
    p = L.probe_order()
    r = np.random.default_rng(4)
    n = 301
    x, y, v = r.random(n) * 0.1 + 0.4, r.random(n) * 0.1 + 0.2, r.uniform(-1, 1, n)
    xc, yc = 0.45, 0.25
    re, im = np.zeros(p), np.zeros(p)
    L.probe_upward_p2e(P(x), P(y), P(v), n, xc, yc, P(re), P(im))
    z = (x - xc) + 1j * (y - yc)
    ref = np.array([-(v * z ** (k + 1)).sum() / (k + 1) for k in range(p)])
    assert rel(re + 1j * im, ref) < 1e-14


@pytest.mark.parametrize("kind", ["potential", "force"])
def test_e2e_matches_shift_formula(kind):
    """upward-kernels.m4:95-149: b_l = sum_c z0^l [-m/l + sum_{k<=l} C(l-1,k-1) a_{k-1} z0^-k]."""
    from math import comb
    L = probe(kind)
    p = L.probe_order()
    r = np.random.default_rng(5)
    x0, y0 = r.uniform(-0.05, 0.05, 4), r.uniform(-0.05, 0.05, 4)
    m = r.uniform(-1, 1, 4)
    a = (r.standard_normal((4, p)) + 1j * r.standard_normal((4, p))) * 0.01 ** np.arange(1, p + 1)
    exps = np.concatenate([np.stack([a[c].real, a[c].imag]) for c in range(4)]).reshape(-1)
    re, im = np.zeros(p), np.zeros(p)
    L.probe_upward_e2e(P(x0), P(y0), P(m), P(np.ascontiguousarray(exps)), P(re), P(im))
    z0 = x0 + 1j * y0
    ref = np.zeros(p, complex)
    for l in range(1, p + 1):
        for c in range(4):
            t = -m[c] / l + sum(comb(l - 1, k - 1) * a[c, k - 1] * z0[c] ** (-k) for k in range(1, l + 1))
            ref[l - 1] += z0[c] ** l * t
    assert rel(re + 1j * im, ref) < 1e-12


def test_potential_kernels_match_formulas():
    """potential-kernels.m4:19-89 (exact64): 0.5 sum v log(r^2 + eps) and
    sum m log(r^2)/2 + Re sum a_{j-1} z^-j."""
    L = probe("potential")
    p = L.probe_order()
    r = np.random.default_rng(6)
    n = 517
    x, y, v = r.random(n), r.random(n), r.uniform(-1, 1, n)
    got = L.probe_potential_p2p(P(x), P(y), P(v), n, 0.3, 0.7)
    eps = 10 * np.finfo(float).eps
    ref = 0.5 * (v * np.log((0.3 - x) ** 2 + (0.7 - y) ** 2 + eps)).sum()
    assert abs(got - ref) < 1e-12 * abs(ref)
    k = 13
    rz, iz, m = r.uniform(1, 2, k), r.uniform(-2, -1, k), r.uniform(-1, 1, k)
    a = r.standard_normal((k, 2, p)) * 0.3 ** np.arange(p)
    got = L.probe_potential_e2p(P(rz), P(iz), P(m), P(np.ascontiguousarray(a.reshape(-1))), k)
    z = rz + 1j * iz
    ref = sum(m[i] * np.log(abs(z[i]) ** 2) / 2 +
              (sum((a[i, 0, j - 1] + 1j * a[i, 1, j - 1]) * z[i] ** (-j) for j in range(1, p + 1))).real
              for i in range(k))
    assert abs(got - ref) < 1e-12 * abs(ref)


def test_force_kernels_match_formulas():
    """force-kernels.m4: P2P, E2P, E2L, L2P on an 8 x 8 brick against their formulas."""
    from math import comb
    L = probe("force")
    p = L.probe_order()
    r = np.random.default_rng(7)
    h = 1e-3
    ix, iy = np.meshgrid(np.arange(8), np.arange(8))
    tx, ty = (0.5 + ix * h).reshape(-1), (0.25 + iy * h).reshape(-1)
    eps = 10 * np.finfo(float).eps
    # P2P
    n = 97
    x, y, v = r.random(n) * 0.02 + 0.49, r.random(n) * 0.02 + 0.24, r.uniform(-1, 1, n)
    xr_, yr_ = np.zeros(64), np.zeros(64)
    L.probe_force_p2p(P(x), P(y), P(v), n, 0.5, 0.25, h, P(xr_), P(yr_))
    dx, dy = tx[:, None] - x[None], ty[:, None] - y[None]
    f = v[None] / (dx * dx + dy * dy + eps)
    assert rel(xr_, (dx * f).sum(1)) < 1e-13 and rel(yr_, (dy * f).sum(1)) < 1e-13
    # E2P: w = m/z - sum (j+1) a_j z^-(j+2); (x, y) += (Re w, -Im w)
    a = (r.standard_normal(p) + 1j * r.standard_normal(p)) * 0.02 ** np.arange(1, p + 1)
    exps = np.ascontiguousarray(np.r_[a.real, a.imag])
    m = 0.7
    xr_, yr_ = np.zeros(64), np.zeros(64)
    L.probe_force_e2p(m, 0.3, -0.2, h, P(exps), P(xr_), P(yr_))
    z = (0.3 + ix * h).reshape(-1) + 1j * (-0.2 + iy * h).reshape(-1)
    w = m / z - sum((j + 1) * a[j] * z ** (-(j + 2)) for j in range(p))
    assert rel(xr_ + 1j * yr_, w.real - 1j * w.imag) < 1e-13
    # E2L + L2P: the local expansion reproduces the multipole field near the brick centre
    k = 5
    x0s, y0s = r.uniform(0.2, 0.3, k), r.uniform(-0.3, -0.2, k)
    ms = r.uniform(0.1, 1, k)
    aa = (r.standard_normal((k, p)) + 1j * r.standard_normal((k, p))) * 0.01 ** np.arange(1, p + 1)
    ex = np.ascontiguousarray(np.concatenate([np.r_[aa[i].real, aa[i].imag] for i in range(k)]))
    rl, il = np.zeros(p + 1), np.zeros(p + 1)
    L.probe_e2l(P(x0s), P(y0s), P(ms), P(ex), k, P(rl), P(il))
    Lc = rl + 1j * il
    z0 = x0s + 1j * y0s
    for l in range(1, p + 1):
        ref = sum(z0[i] ** (-l) * (-ms[i] / l + sum((-1) ** kk * comb(l + kk - 1, kk - 1) * aa[i, kk - 1]
                                                     * z0[i] ** (-kk) for kk in range(1, p + 1)))
                  for i in range(k))
        assert abs(Lc[l] - ref) <= 1e-12 * abs(ref) + 1e-300
    xr_, yr_ = np.zeros(64), np.zeros(64)
    L.probe_l2p(-3.5 * h, -3.5 * h, h, P(rl), P(il), P(xr_), P(yr_))
    zz = (-3.5 * h + ix * h).reshape(-1) + 1j * (-3.5 * h + iy * h).reshape(-1)
    s = sum(l * Lc[l] * zz ** (l - 1) for l in range(1, p + 1))
    assert rel(xr_ + 1j * yr_, s.real - 1j * s.imag) < 1e-13


def test_oracle_potential_passes_reference_verifier():
    """main.cpp:201-262: direct-sum check at tol 1e-8 (theta 0.3, order 12)."""
    w = W.uniform_potential(n=8192, seed=21)
    out = O.potential(0.3, w["xs"], w["ys"], w["vs"], w["xt"], w["yt"], "exact64")
    idx = np.arange(7, len(out), 433)
    ref = O.direct_potential(w["xs"], w["ys"], w["vs"], w["xt"][idx], w["yt"][idx])
    ok, stats = O.check(ref, out[idx], 1e-8)
    assert ok, stats


def test_oracle_force_passes_reference_verifier():
    """main.cpp:201-262 with the force tolerance tol * 100 = 1e-6 (theta 0.5, order 24)."""
    w = W.lamb_oseen_force(n=50000, blocks_per_side=2, h=1.0 / 64, seed=22)
    xo, yo = O.force_mrag(0.5, w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"], "exact64")
    xt, yt = O.mrag_targets(w["x0s"], w["y0s"], w["hs"])
    idx = np.arange(7, len(xo), 433)
    rx, ry = O.direct_force(w["xs"], w["ys"], w["vs"], xt[idx], yt[idx])
    assert O.check(rx, xo[idx], 1e-6)[0]
    assert O.check(ry, yo[idx], 1e-6)[0]


def exact_topology(keys, leafcap):
    """Breadth-first topology from sorted keys with exact bounds (upward.cpp:223-277):
    (level, cx, cy, s, e, inner) per node."""
    out = []
    q = [(0, 0, 0, 0, 0, len(keys))]
    n = len(keys)
    while q:
        nq = []
        for (l, x, y, mask, s, e) in q:
            inner = e - s > leafcap and l + 1 <= 15
            out.append((l, x, y, s, e, inner))
            if inner:
                shift = 2 * (15 - l - 1)
                for c in range(4):
                    k1 = mask | (c << shift)
                    lo = s if c == 0 else s + int(np.searchsorted(keys[s:e], k1, "left"))
                    hi = e if c == 3 else s + int(np.searchsorted(keys[s:e], k1 + (1 << shift) - 1, "right"))
                    nq.append((l + 1, 2 * x + (c & 1), 2 * y + (c >> 1), k1, lo, hi))
        q = nq
    return np.array(out, dtype=np.int64)


@pytest.mark.parametrize("case", ["potential_uniform", "force_lamb_oseen", "potential_coincident_cluster"])
def test_oracle_topology_is_exact_bound_topology(case):
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", f"{case}.npz"))
    kind = str(z["kind"])
    keys = O.sort_sources(z["xs"], z["ys"], z["vs"], kind, "exact64")[0]
    topo = exact_topology(keys, O.LEAF[kind])
    t = O.canonical(O.tree(z["xs"], z["ys"], z["vs"], kind, "exact64"))
    assert len(topo) == len(t["level"])
    for col, k in enumerate(("level", "cx", "cy", "s", "e")):
        assert np.array_equal(topo[:, col], t[k]), k
    assert np.array_equal(topo[:, 5].astype(bool), t["inner"])


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_golden_fixture_reproduced(path):
    """The committed fixtures are outputs of this oracle build: re-running it gives them back
    bit for bit (pins the oracle build used by the GPU parity tests)."""
    z = np.load(path)
    kind = str(z["kind"])
    keys, xs, ys, vs, bbox = O.sort_sources(z["xs"], z["ys"], z["vs"], kind, "exact64")
    assert np.array_equal(keys, z["keys"]) and np.array_equal(xs, z["sorted_x"])
    assert np.array_equal(bbox, z["frame"])
    t = O.canonical(O.tree(z["xs"], z["ys"], z["vs"], kind, "exact64"))
    for k in ("level", "cx", "cy", "s", "e", "inner", "mass", "xcom", "ycom", "r", "exps"):
        assert np.array_equal(t[k], z[f"tree_{k}"]), k
    theta = float(z["theta"])
    if kind == "potential":
        out = O.potential(theta, z["xs"], z["ys"], z["vs"], z["xt"], z["yt"], "exact64")
        assert np.array_equal(out, z["potential_exact64"])
    else:
        xo, yo = O.force_mrag(theta, z["xs"], z["ys"], z["vs"], z["x0s"], z["y0s"], z["hs"], "exact64")
        assert np.array_equal(xo, z["xforce_exact64"]) and np.array_equal(yo, z["yforce_exact64"])


def test_faithful_mode_differs_only_by_float_constants():
    """The float-typed literals / single-precision log of the reference's ISPC kernels move the
    result by far less than the treecode's own truncation error, but measurably."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "potential_uniform.npz"))
    d = rel(z["potential_faithful"], z["potential_exact64"])
    assert 0 < d < 1e-6
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "force_lamb_oseen.npz"))
    d = rel(z["xforce_faithful"], z["xforce_exact64"])
    assert 0 < d < 1e-6
