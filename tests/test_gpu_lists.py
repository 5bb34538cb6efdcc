"""The interaction lists are built in one walk into per-warp scratch runs sized from what
earlier solves on the context needed; a run that outgrows its region makes the solve fall
back to a second walk (and the regions grow).  A fresh context's first solve of a large-list
problem takes the fallback and the next one the copy: both give the same result bit for bit,
and so does a third after a smaller problem has run in between."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "2d-treecodes_b200"))

import treecodes as T      # noqa: E402
import workloads as W      # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_potential_lists_fallback_and_copy_agree(precision):
    w = W.gaussian_mixture_potential(n=1 << 17)
    small = W.uniform_potential(n=5000)
    ctx = T.Context(device=0, precision=precision)
    try:
        outs, walks = [], []
        for it in range(3):
            outs.append(ctx.potential_host(0.3, w["xs"], w["ys"], w["vs"], w["xt"], w["yt"]))
            walks.append(ctx.stats()["list_walks"])
            if it == 1:
                ctx.potential_host(0.5, small["xs"], small["ys"], small["vs"], small["xt"],
                                   small["yt"])
        assert walks == [2, 1, 1]
        assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    finally:
        ctx.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_force_lists_fallback_and_copy_agree(precision):
    w = W.vortex_sheet_force(n=1 << 18, blocks_per_side=8)
    ctx = T.Context(device=0, precision=precision)
    try:
        a = ctx.force_mrag_host(0.3, w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"])
        wa = ctx.stats()["list_walks"]
        b = ctx.force_mrag_host(0.3, w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"])
        assert (wa, ctx.stats()["list_walks"]) == (2, 1)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    finally:
        ctx.close()
