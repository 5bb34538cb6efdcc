"""Full-size parity of the two large benchmark workloads against the oracle (the reference's
own drivers in EXACT64 mode, node capacity raised so they do not overflow at these sizes).

* 16,777,216-source vortex sheet, 4096 blocks of 32 x 32 targets, theta 0.5: bounding square,
  Morton keys, permutation, sorted sources and the whole tree (ranges, levels, cells, mass,
  centre of mass, radius) bit-exact; expansions within 1e-12; forces within 1e-12 relative L2
  on every 16th block (256 blocks, 262,144 targets).  The reference evaluates exactly the
  blocks it is given (drivers/treecode-force.cpp:219-225), so the oracle runs on those blocks
  alone with the tree of all sources.
* 4,194,304-source Gaussian mixture, targets a copy of the sources, theta 0.3 / 0.5 / 0.7: tree
  bit-exact, potentials within 1e-12 relative L2 on every 512th target (8192 targets); the
  reference evaluates each target on its own (drivers/treecode-potential.cpp:101-102).  The
  mixed form stays within 1e-6 of the FP64 direct sum and of the plain form at every theta.
"""
import numpy as np
import pytest
import torch

import oracle as O
import workloads as W
from tc_helpers import dev, dev_empty, host, rel_l2
from test_gpu_parity import assert_tree_matches, gpu_tree

pytestmark = pytest.mark.gpu

TOL = 1e-12
TOL_MIXED = 1e-6
BLOCK_STRIDE = 16
TARGET_STRIDE = 512


def tree_check_big(ctx, kind, w):
    keys, xs, ys, vs, frame = O.sort_sources(w["xs"], w["ys"], w["vs"], kind, "exact64_big")
    ref = O.canonical(O.tree(w["xs"], w["ys"], w["vs"], kind, "exact64_big"))
    g, cn = gpu_tree(ctx, kind, w)
    assert_tree_matches(g, cn, keys, (xs, ys, vs), frame, ref, w["xs"])
    return len(cn["level"])


@pytest.fixture(scope="module")
def sheet():
    return W.vortex_sheet_force()


@pytest.fixture(scope="module")
def mixture():
    return W.gaussian_mixture_potential()


def test_vortex_sheet_tree_full_size(gpu_ctx, sheet):
    assert len(sheet["xs"]) == 1 << 24 and len(sheet["x0s"]) == 4096
    nodes = tree_check_big(gpu_ctx, "force", sheet)
    assert nodes > 8e4   # beyond the reference's fixed node capacity


def test_vortex_sheet_forces_full_size_sampled(gpu_ctx, sheet):
    w = sheet
    nb = len(w["x0s"])
    d = {k: dev(w[k]) for k in ("xs", "ys", "vs", "x0s", "y0s", "hs")}
    xo, yo = dev_empty(nb * 1024), dev_empty(nb * 1024)
    gpu_ctx.force_mrag_device(w["theta"], d["xs"], d["ys"], d["vs"], d["x0s"], d["y0s"], d["hs"],
                              xo, yo)
    blocks = np.arange(3, nb, BLOCK_STRIDE)
    rx, ry = O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"][blocks],
                          w["y0s"][blocks], w["hs"][blocks], "exact64_big")
    gx = host(xo).reshape(nb, 1024)[blocks].ravel()
    gy = host(yo).reshape(nb, 1024)[blocks].ravel()
    assert rel_l2(np.r_[gx, gy], np.r_[rx, ry]) < TOL


def test_gaussian_mixture_tree_full_size(gpu_ctx, mixture):
    assert len(mixture["xs"]) == 1 << 22
    tree_check_big(gpu_ctx, "potential", mixture)


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_gaussian_mixture_potential_full_size_sampled(gpu_ctx, mixture, theta):
    w = mixture
    m = len(w["xt"])
    d = {k: dev(w[k]) for k in ("xs", "ys", "vs", "xt", "yt")}
    outs = {}
    for prec in (0, 1):
        gpu_ctx.set_precision(prec)
        try:
            out = dev_empty(m)
            gpu_ctx.potential_device(theta, d["xs"], d["ys"], d["vs"], d["xt"], d["yt"], out)
        finally:
            gpu_ctx.set_precision(0)
        outs[prec] = out
    idx = np.arange(5, m, TARGET_STRIDE)
    ref = O.potential(theta, w["xs"], w["ys"], w["vs"], w["xt"][idx], w["yt"][idx],
                      "exact64_big")
    assert rel_l2(host(outs[0])[idx], ref) < TOL

    # the mixed form: within 1e-6 of the plain form everywhere, and of the FP64 direct sum on
    # the sample beyond the treecode's own truncation error
    err_plain = float((outs[1] - outs[0]).norm() / outs[0].norm())
    assert err_plain < TOL_MIXED, err_plain
    ti = torch.as_tensor(idx, device="cuda")
    direct = dev_empty(len(idx))
    gpu_ctx.direct_potential_device(d["xs"], d["ys"], d["vs"], d["xt"][ti], d["yt"][ti], direct)
    e64 = float((outs[0][ti] - direct).norm() / direct.norm())
    e32 = float((outs[1][ti] - direct).norm() / direct.norm())
    assert e32 < e64 + TOL_MIXED, (e32, e64)
