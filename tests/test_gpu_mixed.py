"""GPU checks of the mixed-precision form (FP32 P2P and multipole series with compensated
sums; FP64 bounding box, keys, tree, upward pass, local expansions and monopole logs).

It is gated on accuracy, not on bits: at most 1e-6 relative L2 error against the FP64 direct sum,
and against the plain FP64 GPU form on the same inputs, on the benchmark workloads."""
import numpy as np
import pytest
import torch

import workloads as W
from tc_helpers import dev, dev_empty, host, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-6


def run_force(ctx, w, precision, theta=None):
    theta = w["theta"] if theta is None else theta
    d = {k: dev(w[k]) for k in ("xs", "ys", "vs", "x0s", "y0s", "hs")}
    m = len(w["x0s"]) * 1024
    xo, yo = dev_empty(m), dev_empty(m)
    ctx.set_precision(precision)
    try:
        ctx.force_mrag_device(theta, d["xs"], d["ys"], d["vs"], d["x0s"], d["y0s"], d["hs"], xo, yo)
    finally:
        ctx.set_precision(0)
    return d, xo, yo


def direct_force_sample(ctx, d, m, nsample=2048):
    idx = torch.arange(7, m, max(1, m // nsample), device="cuda")[:nsample]
    ib, rem = idx // 1024, idx % 1024
    xt = d["x0s"][ib] + (rem % 32).double() * d["hs"][ib]
    yt = d["y0s"][ib] + (rem // 32).double() * d["hs"][ib]
    rx, ry = dev_empty(len(idx)), dev_empty(len(idx))
    ctx.direct_force_device(d["xs"], d["ys"], d["vs"], xt, yt, rx, ry)
    return idx, torch.cat([rx, ry])


@pytest.mark.parametrize("name", ["lamb_oseen_force", "vortex_sheet_force"])
def test_mixed_force_accuracy(gpu_ctx, name):
    w = W.WORKLOADS[name]()
    d, xm, ym = run_force(gpu_ctx, w, 1)
    _, x64, y64 = run_force(gpu_ctx, w, 0)
    m = xm.numel()
    idx, ref = direct_force_sample(gpu_ctx, d, m)
    err_direct = float((torch.cat([xm[idx], ym[idx]]) - ref).norm() / ref.norm())
    err_plain = float((torch.cat([xm, ym]) - torch.cat([x64, y64])).norm() / torch.cat([x64, y64]).norm())
    assert err_direct < TOL, err_direct
    assert err_plain < TOL, err_plain


def test_mixed_force_small_cases(gpu_ctx):
    """Mixed form against the plain form on small, clustered and negligible-weight inputs."""
    import glob
    import os
    for path in sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "force_*.npz"))):
        z = np.load(path)
        w = {k: z[k] for k in z.files}
        w["theta"] = float(z["theta"])
        _, xm, ym = run_force(gpu_ctx, w, 1)
        ref = np.r_[z["xforce_exact64"], z["yforce_exact64"]]
        assert rel_l2(np.r_[host(xm), host(ym)], ref) < TOL, path


@pytest.mark.parametrize("name", ["uniform_potential", "gaussian_mixture_potential"])
def test_mixed_potential_accuracy(gpu_ctx, name):
    w = W.WORKLOADS[name]() if name == "uniform_potential" else W.gaussian_mixture_potential(n=1 << 20)
    d = {k: dev(w[k]) for k in ("xs", "ys", "vs", "xt", "yt")}
    m = len(w["xt"])
    outs = {}
    for prec in (0, 1):
        gpu_ctx.set_precision(prec)
        out = dev_empty(m)
        gpu_ctx.potential_device(w["theta"], d["xs"], d["ys"], d["vs"], d["xt"], d["yt"], out)
        outs[prec] = out
    gpu_ctx.set_precision(0)
    err_plain = float((outs[1] - outs[0]).norm() / outs[0].norm())
    assert err_plain < TOL, err_plain
    idx = torch.arange(7, m, max(1, m // 2048), device="cuda")[:2048]
    ref = dev_empty(len(idx))
    gpu_ctx.direct_potential_device(d["xs"], d["ys"], d["vs"], d["xt"][idx], d["yt"][idx], ref)
    e64 = float((outs[0][idx] - ref).norm() / ref.norm())
    e32 = float((outs[1][idx] - ref).norm() / ref.norm())
    # the mixed form adds at most 1e-6 to the treecode's own truncation error
    assert e32 < e64 + TOL, (e32, e64)


def test_mixed_is_deterministic(gpu_ctx):
    w = W.lamb_oseen_force(n=1 << 18, blocks_per_side=8, h=1.0 / 256)
    _, x1, y1 = run_force(gpu_ctx, w, 1)
    _, x2, y2 = run_force(gpu_ctx, w, 1)
    assert torch.equal(x1, x2) and torch.equal(y1, y2)
