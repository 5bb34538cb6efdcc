"""GPU parity: the CUDA path (through the C ABI) against the oracle -- the reference's own
drivers compiled on the CPU with the restated kernels in exact64 mode.

Gates:
  * Morton keys, sorted sources, permutation and tree topology bit-exact;
  * node mass, centre of mass and radius bit-exact (the far/near decisions depend on them);
  * expansions, potentials and forces within 1e-12 relative L2 (FP64 plain form).
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
import treecodes as T
import workloads as W
from tc_helpers import dev, dev_empty, gpu_force, gpu_potential, host, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def gpu_tree(ctx, kind, w):
    g = ctx.tree(kind, dev(w["xs"]), dev(w["ys"]), dev(w["vs"]))
    cn = O.canonical(dict(s=g["s"], e=g["e"], inner=g["inner"], child=g["child"], mass=g["mass"],
                          xcom=g["xcom"], ycom=g["ycom"], r=g["r"], exps=g["exps"]))
    return g, cn


def assert_tree_matches(g, cn, ref_keys, ref_sorted, ref_frame, ref_tree, xs_in):
    assert np.array_equal(g["frame"], ref_frame)
    assert np.array_equal(g["keys"], ref_keys)
    for got, ref in zip((g["xs"], g["ys"], g["vs"]), ref_sorted):
        assert np.array_equal(got, ref)
    assert np.array_equal(xs_in[g["perm"]], g["xs"])
    assert len(cn["level"]) == len(ref_tree["level"])
    for k in ("level", "cx", "cy", "s", "e", "inner", "mass", "xcom", "ycom", "r"):
        assert np.array_equal(cn[k], ref_tree[k]), k
    assert rel_l2(cn["exps"], ref_tree["exps"]) < TOL


# ------------------------------------------------------------------------- golden fixtures
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_golden_fixture(gpu_ctx, path):
    z = np.load(path)
    kind = str(z["kind"])
    w = {k: z[k] for k in z.files}
    g, cn = gpu_tree(gpu_ctx, kind, w)
    ref_tree = {k: z[f"tree_{k}"] for k in ("level", "cx", "cy", "s", "e", "inner", "mass",
                                             "xcom", "ycom", "r", "exps")}
    assert_tree_matches(g, cn, z["keys"], (z["sorted_x"], z["sorted_y"], z["sorted_v"]),
                        z["frame"], ref_tree, z["xs"])
    theta = float(z["theta"])
    if kind == "potential":
        out = gpu_potential(gpu_ctx, w, theta)
        assert rel_l2(out, z["potential_exact64"]) < TOL
        assert rel_l2(out, z["potential_faithful"]) < 1e-6
    else:
        xo, yo = gpu_force(gpu_ctx, w, theta)
        assert rel_l2(np.r_[xo, yo], np.r_[z["xforce_exact64"], z["yforce_exact64"]]) < TOL
        assert rel_l2(np.r_[xo, yo], np.r_[z["xforce_faithful"], z["yforce_faithful"]]) < 1e-6


# ------------------------------------------------------------------------- live oracle
def live_tree_check(ctx, kind, w):
    keys, xs, ys, vs, frame = O.sort_sources(w["xs"], w["ys"], w["vs"], kind, "exact64")
    ref = O.canonical(O.tree(w["xs"], w["ys"], w["vs"], kind, "exact64"))
    g, cn = gpu_tree(ctx, kind, w)
    assert_tree_matches(g, cn, keys, (xs, ys, vs), frame, ref, w["xs"])


def test_uniform_potential_full_size(gpu_ctx):
    """N = M = 65,536 uniform sources, targets a copy of the sources, theta 0.5."""
    w = W.uniform_potential()
    live_tree_check(gpu_ctx, "potential", w)
    ref = O.potential(w["theta"], w["xs"], w["ys"], w["vs"], w["xt"], w["yt"], "exact64")
    assert rel_l2(gpu_potential(gpu_ctx, w), ref) < TOL


def test_lamb_oseen_force_full_size(gpu_ctx):
    """1,048,576 Lamb-Oseen sources, 1024 blocks of 32 x 32 targets, theta 0.5."""
    w = W.lamb_oseen_force()
    live_tree_check(gpu_ctx, "force", w)
    rx, ry = O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"],
                          "exact64")
    xo, yo = gpu_force(gpu_ctx, w)
    assert rel_l2(np.r_[xo, yo], np.r_[rx, ry]) < TOL


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_gaussian_mixture_potential_theta_sweep(gpu_ctx, theta):
    """A quarter-million-source mixture, every target compared (the full-size 4M mixture is
    compared on a target sample in test_gpu_fullsize.py)."""
    w = W.gaussian_mixture_potential(n=1 << 18)
    if theta == 0.5:
        live_tree_check(gpu_ctx, "potential", w)
    ref = O.potential(theta, w["xs"], w["ys"], w["vs"], w["xt"], w["yt"], "exact64")
    assert rel_l2(gpu_potential(gpu_ctx, w, theta), ref) < TOL


def test_vortex_sheet_force_reduced(gpu_ctx):
    """The vortex sheet at 1M sources and 16 x 16 blocks (h = 1/512): oracle-size case."""
    w = W.vortex_sheet_force(n=1 << 20, blocks_per_side=16, h=1.0 / 512)
    live_tree_check(gpu_ctx, "force", w)
    rx, ry = O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"],
                          "big")
    ex, ey = O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"],
                          "exact64")
    xo, yo = gpu_force(gpu_ctx, w)
    assert rel_l2(np.r_[xo, yo], np.r_[ex, ey]) < TOL
    assert rel_l2(np.r_[xo, yo], np.r_[rx, ry]) < 1e-6


# ------------------------------------------------------------------------- edge cases
@pytest.mark.parametrize("n", [1, 2, 5, 192, 193, 512, 513])
def test_small_source_counts(gpu_ctx, n):
    r = np.random.default_rng(n)
    w = dict(xs=r.random(n), ys=r.random(n), vs=r.uniform(-1, 1, n))
    w["xt"], w["yt"] = r.random(37), r.random(37)
    ref = O.potential(0.5, w["xs"], w["ys"], w["vs"], w["xt"], w["yt"], "exact64")
    assert rel_l2(gpu_potential(gpu_ctx, w, 0.5), ref) < TOL
    w.update(x0s=np.array([0.1, 0.5]), y0s=np.array([0.2, 0.6]), hs=np.array([0.01, 0.005]))
    rx, ry = O.force_mrag(0.5, w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"], "exact64")
    xo, yo = gpu_force(gpu_ctx, w, 0.5)
    assert rel_l2(np.r_[xo, yo], np.r_[rx, ry]) < TOL


@pytest.mark.parametrize("n", [2047, 2049, 3071, 3072, 3073, 6145, 16385])
def test_sort_tile_boundaries_and_host_path(gpu_ctx, n):
    """Source counts at the radix passes' tile edges (3072 items) and the gather's (2048):
    keys, sorted sources, permutation and tree bit-exact with the oracle (device path, values
    resident); the host entry point, whose sort gathers x and y before v arrives, gives the
    device path's outputs bit for bit."""
    r = np.random.default_rng(n)
    w = dict(xs=r.random(n), ys=r.random(n), vs=r.uniform(-1, 1, n))
    live_tree_check(gpu_ctx, "potential", w)
    w["xt"], w["yt"] = r.random(300), r.random(300)
    out = gpu_potential(gpu_ctx, w, 0.5)
    assert np.array_equal(gpu_ctx.potential_host(0.5, w["xs"], w["ys"], w["vs"], w["xt"],
                                                 w["yt"]), out)
    w.update(x0s=np.array([0.1, 0.5]), y0s=np.array([0.2, 0.6]), hs=np.array([0.01, 0.005]))
    xo, yo = gpu_force(gpu_ctx, w, 0.5)
    hx, hy = gpu_ctx.force_mrag_host(0.5, w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"])
    assert np.array_equal(hx, xo) and np.array_equal(hy, yo)


def test_zero_sources_give_zero_output(gpu_ctx):
    e = np.zeros(0)
    out = gpu_ctx.potential_host(0.5, e, e, e, np.array([0.1, 0.2]), np.array([0.3, 0.4]))
    assert np.array_equal(out, [0.0, 0.0])
    xo, yo = gpu_ctx.force_mrag_host(0.5, e, e, e, np.array([0.0]), np.array([0.0]), np.array([0.1]))
    assert not xo.any() and not yo.any()


def test_targets_outside_sources_and_ragged_groups(gpu_ctx):
    r = np.random.default_rng(9)
    n = 20000
    w = dict(xs=r.random(n), ys=r.random(n), vs=r.uniform(-1, 1, n))
    w["xt"] = np.r_[r.uniform(-3, 4, 1001), r.random(30)]
    w["yt"] = np.r_[r.uniform(-3, 4, 1001), r.random(30)]
    ref = O.potential(0.5, w["xs"], w["ys"], w["vs"], w["xt"], w["yt"], "exact64")
    assert rel_l2(gpu_potential(gpu_ctx, w, 0.5), ref) < TOL


@pytest.mark.parametrize("theta", [0.2, 1.0])
def test_force_theta_extremes(gpu_ctx, theta):
    w = W.lamb_oseen_force(n=200000, blocks_per_side=4, h=1.0 / 128, seed=31)
    rx, ry = O.force_mrag(theta, w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"], "exact64")
    xo, yo = gpu_force(gpu_ctx, w, theta)
    assert rel_l2(np.r_[xo, yo], np.r_[rx, ry]) < TOL


def test_blocks_with_individual_spacings(gpu_ctx):
    """MRAG blocks of different resolutions, overlapping each other and the sources."""
    w = W.lamb_oseen_force(n=300000, blocks_per_side=1, seed=32)
    r = np.random.default_rng(32)
    nb = 37
    w["x0s"], w["y0s"] = r.uniform(0.2, 0.7, nb), r.uniform(0.2, 0.7, nb)
    w["hs"] = 2.0 ** -r.integers(6, 12, nb)
    rx, ry = O.force_mrag(0.5, w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"], "exact64")
    xo, yo = gpu_force(gpu_ctx, w, 0.5)
    assert rel_l2(np.r_[xo, yo], np.r_[rx, ry]) < TOL


def test_reference_entry_points(gpu_ctx):
    """The reference-compatible host entry points give the device-path results."""
    w = W.lamb_oseen_force(n=50000, blocks_per_side=2, h=1.0 / 64, seed=33)
    xo, yo = T.treecode_force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"])
    gx, gy = gpu_force(gpu_ctx, w)
    assert np.array_equal(xo, gx) and np.array_equal(yo, gy)
    w = W.uniform_potential(n=9000, seed=34)
    out = T.treecode_potential(w["theta"], w["xs"], w["ys"], w["vs"], w["xt"], w["yt"])
    assert np.array_equal(out, gpu_potential(gpu_ctx, w))


def test_invalid_arguments_report_status(gpu_ctx):
    rc = gpu_ctx.lib.tc_potential_device(gpu_ctx.h, 0.5, None, None, None, -5, None, None, 10, None)
    assert rc == 1 and T.last_status() == 1          # TC_ERR_INVALID
    with pytest.raises(T.TreecodeError):
        T._check(gpu_ctx.lib.tc_force_mrag_device(gpu_ctx.h, 0.5, None, None, None, 10, None,
                                                  None, None, -1, None, None))


# ------------------------------------------------------------------------- full-size properties
def test_vortex_sheet_full_size_properties(gpu_ctx):
    """16,777,216 sources, 4096 blocks: too large for the CPU oracle, so checked through
    size-independent properties: accuracy against the FP64 direct sum on a strided subsample,
    exact linearity under v -> 2v (all arithmetic scales by a power of two), and run-to-run
    determinism."""
    import torch
    w = W.vortex_sheet_force()
    d = {k: dev(w[k]) for k in ("xs", "ys", "vs", "x0s", "y0s", "hs")}
    m = len(w["x0s"]) * 1024

    def run(vs):
        xo, yo = dev_empty(m), dev_empty(m)
        gpu_ctx.force_mrag_device(0.5, d["xs"], d["ys"], vs, d["x0s"], d["y0s"], d["hs"], xo, yo)
        return xo, yo

    xo, yo = run(d["vs"])
    x2, y2 = run(d["vs"])
    assert torch.equal(xo, x2) and torch.equal(yo, y2)
    x3, y3 = run(2.0 * d["vs"])
    assert torch.equal(x3, 2.0 * xo) and torch.equal(y3, 2.0 * yo)
    idx = torch.arange(7, m, 433 * 4, device="cuda")
    ib, rem = idx // 1024, idx % 1024
    xt = d["x0s"][ib] + (rem % 32).double() * d["hs"][ib]
    yt = d["y0s"][ib] + (rem // 32).double() * d["hs"][ib]
    rx, ry = dev_empty(len(idx)), dev_empty(len(idx))
    gpu_ctx.direct_force_device(d["xs"], d["ys"], d["vs"], xt, yt, rx, ry)
    err = rel_l2(np.r_[host(xo[idx]), host(yo[idx])], np.r_[host(rx), host(ry)])
    assert err < 1e-9


def test_gpu_direct_sum_matches_cpu_direct_sum(gpu_ctx):
    """Pins the GPU direct sum used for full-size accuracy against main.cpp's CPU direct sum."""
    w = W.vortex_sheet_force(n=1 << 20, blocks_per_side=2)
    r = np.random.default_rng(35)
    xt, yt = r.random(64), r.random(64)
    cx, cy = O.direct_force(w["xs"], w["ys"], w["vs"], xt, yt)
    gx, gy = dev_empty(64), dev_empty(64)
    gpu_ctx.direct_force_device(dev(w["xs"]), dev(w["ys"]), dev(w["vs"]), dev(xt), dev(yt), gx, gy)
    assert rel_l2(np.r_[host(gx), host(gy)], np.r_[cx, cy]) < 1e-12
    cp = O.direct_potential(w["xs"], w["ys"], w["vs"], xt, yt)
    gp = dev_empty(64)
    gpu_ctx.direct_potential_device(dev(w["xs"]), dev(w["ys"]), dev(w["vs"]), dev(xt), dev(yt), gp)
    assert rel_l2(host(gp), cp) < 1e-12


def test_potential_log_within_a_few_ulp_of_the_library(gpu_ctx):
    """The potential kernels' own logarithm (log_pos: table-driven reduction and log1p series)
    against CUDA's log on 2^20 arguments spanning the range the kernels feed it (r^2 + 10 eps
    from ~2e-15 up, far-cell |z|^2), plus arguments next to 1, to powers of two and to the
    sqrt(2) split of the reduction."""
    r = np.random.default_rng(5)
    x = np.exp(r.uniform(np.log(2e-15), np.log(1e6), 1 << 20))
    edges = []
    for b in [1.0, 2.0, 0.5, 2.0 ** -40, 2.0 ** 19, np.sqrt(2.0), np.sqrt(0.5)]:
        edges += [b, np.nextafter(b, 0), np.nextafter(b, 4 * b)]
        edges += list(b * (1 + np.linspace(-1e-6, 1e-6, 101)))
    x = np.r_[x, np.array(edges)]
    xd = dev(x)
    out = dev_empty(2 * len(x))
    gpu_ctx.log_probe_device(xd, out)
    o = host(out).reshape(-1, 2)
    mine, lib = o[:, 0], o[:, 1]
    ulp = np.spacing(np.abs(lib))
    err = np.abs(mine - lib)
    assert np.all(err <= 4 * ulp), (err / ulp).max()


def test_force_host_outputs_copied_in_runs(gpu_ctx):
    """Host outputs of 2^21 targets or more come back in runs of blocks copied while later runs
    are evaluated: the same values as the device entry point, bit for bit, both precisions."""
    w = W.lamb_oseen_force(n=100000, blocks_per_side=48, h=1.0 / (32 * 48))   # 2304 blocks
    for precision in (0, 1):
        gpu_ctx.set_precision(precision)
        try:
            hx, hy = gpu_ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"],
                                             w["y0s"], w["hs"])
            dx, dy = gpu_force(gpu_ctx, w)
        finally:
            gpu_ctx.set_precision(0)
        assert np.array_equal(hx, dx) and np.array_equal(hy, dy)


def test_timing_modes_give_the_same_results(gpu_ctx):
    """Phase timing (mode 1) and the per-kernel measurement mode (2, the force's near and far
    field one after the other) change the scheduling only: the outputs are bit-identical."""
    w = W.lamb_oseen_force(n=120000, blocks_per_side=4, h=1.0 / 128, seed=36)
    ref = {}
    for precision in (0, 1):
        gpu_ctx.set_precision(precision)
        try:
            for mode in (0, 1, 2):
                gpu_ctx.set_timing(mode)
                got = gpu_force(gpu_ctx, w)
                if mode == 0:
                    ref[precision] = got
                else:
                    assert np.array_equal(got[0], ref[precision][0])
                    assert np.array_equal(got[1], ref[precision][1])
                if mode == 2:
                    st = gpu_ctx.stats()
                    assert 0 < st["far_kernel_ms"] < st["eval_kernel_ms"]
        finally:
            gpu_ctx.set_timing(0)
            gpu_ctx.set_precision(0)


def test_launch_overlap_changes_nothing(gpu_ctx):
    """Programmatic dependent launch of the sort, tree and upward kernel chains (the default) and
    plain launches give the same outputs, bit for bit, for both entry points (device and host
    pointers) and both forms; the sizes cover several radix tiles, tree levels and E2E
    launches."""
    wp = W.gaussian_mixture_potential(n=200000)
    wf = W.lamb_oseen_force(n=300000, blocks_per_side=16, h=1.0 / 512)
    try:
        for precision in (0, 1):
            gpu_ctx.set_precision(precision)
            outs = []
            for overlap in (True, False):
                gpu_ctx.set_launch_overlap(overlap)
                p = gpu_potential(gpu_ctx, wp, 0.5)
                xo, yo = gpu_force(gpu_ctx, wf, 0.5)
                # the host entry points sort with the values arriving late (another chain)
                hp = gpu_ctx.potential_host(0.5, wp["xs"], wp["ys"], wp["vs"], wp["xt"], wp["yt"])
                hx, hy = gpu_ctx.force_mrag_host(0.5, wf["xs"], wf["ys"], wf["vs"], wf["x0s"],
                                                 wf["y0s"], wf["hs"])
                outs.append((p, xo, yo, hp, hx, hy))
            for a, b in zip(*outs):
                assert np.array_equal(a, b)
    finally:
        gpu_ctx.set_launch_overlap(True)
        gpu_ctx.set_precision(0)
