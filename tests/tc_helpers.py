"""Shared helpers of the test-suite: device transfers and error norms."""
import numpy as np


def dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def dev_empty(n):
    import torch
    return torch.empty(int(n), dtype=torch.float64, device="cuda")


def host(t):
    return t.detach().cpu().numpy()


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


def gpu_potential(ctx, w, theta=None):
    theta = w["theta"] if theta is None else theta
    out = dev_empty(len(w["xt"]))
    ctx.potential_device(theta, dev(w["xs"]), dev(w["ys"]), dev(w["vs"]), dev(w["xt"]),
                         dev(w["yt"]), out)
    return host(out)


def gpu_force(ctx, w, theta=None):
    theta = w["theta"] if theta is None else theta
    nt = len(w["x0s"]) * 1024
    xo, yo = dev_empty(nt), dev_empty(nt)
    ctx.force_mrag_device(theta, dev(w["xs"]), dev(w["ys"]), dev(w["vs"]), dev(w["x0s"]),
                          dev(w["y0s"]), dev(w["hs"]), xo, yo)
    return host(xo), host(yo)
