"""Runtime-selected expansion orders (tc_set_orders) and MRAG block sides (tc_set_blocksize),
the reference's build-time potential-order / force-order / mrag-blocksize: at each order the
oracle is built for (8, 16, 28) and each block side (16, 64) the plain form matches the
reference drivers built with that setting (EXACT64 kernels) to 1e-12 relative L2, the mixed
form stays within 1e-6 of the plain one, and unsupported settings are refused."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [os.path.join(ROOT, "2d-treecodes_b200"), os.path.join(ROOT, "oracle")]

import treecodes as T      # noqa: E402
import workloads as W      # noqa: E402

pytestmark = pytest.mark.gpu

ORACLE_ORDERS = (8, 16, 28)


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def force_case():
    return W.lamb_oseen_force(n=30000, blocks_per_side=2, h=1.0 / 64)


@pytest.fixture(scope="module")
def potential_case():
    return W.uniform_potential(n=30000)


@pytest.mark.parametrize("order", ORACLE_ORDERS)
def test_force_order_matches_reference_build(force_case, order):
    import oracle as O
    w = force_case
    ctx = T.Context(device=0)
    try:
        ctx.set_orders(T.ORDER_POTENTIAL, order)
        xo, yo = ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"],
                                     w["hs"])
        rx, ry = O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"],
                              mode=f"exact64_o{order}")
        assert rel_l2(np.r_[xo, yo], np.r_[rx, ry]) < 1e-12
        ctx.set_precision(1)
        mx, my = ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"],
                                     w["hs"])
        assert rel_l2(np.r_[mx, my], np.r_[xo, yo]) < 1e-6
    finally:
        ctx.close()


@pytest.mark.parametrize("order", ORACLE_ORDERS)
def test_potential_order_matches_reference_build(potential_case, order):
    import oracle as O
    w = potential_case
    ctx = T.Context(device=0)
    try:
        ctx.set_orders(order, T.ORDER_FORCE)
        out = ctx.potential_host(w["theta"], w["xs"], w["ys"], w["vs"], w["xt"], w["yt"])
        ref = O.potential(w["theta"], w["xs"], w["ys"], w["vs"], w["xt"], w["yt"],
                          mode=f"exact64_o{order}")
        assert rel_l2(out, ref) < 1e-12
        ctx.set_precision(1)
        mixed = ctx.potential_host(w["theta"], w["xs"], w["ys"], w["vs"], w["xt"], w["yt"])
        assert rel_l2(mixed, out) < 1e-6
    finally:
        ctx.close()


def test_every_supported_order_runs_and_converges(force_case):
    """The force error against the direct sum falls with the order (theta 0.5)."""
    w = force_case
    ctx = T.Context(device=0)
    try:
        sample = np.arange(7, len(w["x0s"]) * 1024, 433)
        import datasets as D
        xt, yt = D.block_targets(w["x0s"], w["y0s"], w["hs"])
        du, dv = D.direct_force(w["xs"], w["ys"], w["vs"], xt[sample], yt[sample])
        errs = []
        for p in T.supported_orders():
            ctx.set_orders(T.ORDER_POTENTIAL, p)
            xo, yo = ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"],
                                         w["y0s"], w["hs"])
            errs.append(rel_l2(np.r_[xo[sample], yo[sample]], np.r_[du, dv]))
        assert all(b < a for a, b in zip(errs[:3], errs[1:4])), errs   # 4 < 8 < 12 < 16
        assert errs[-1] < 1e-9, errs
    finally:
        ctx.close()


def test_unsupported_orders_are_refused():
    assert T.supported_orders() == [4, 8, 12, 16, 20, 24, 28]
    ctx = T.Context(device=0)
    try:
        for bad in ((10, 24), (12, 32), (0, 24), (12, -4)):
            with pytest.raises(T.TreecodeError, match="order"):
                ctx.set_orders(*bad)
        # a refused setting leaves the orders as they were: the defaults still solve
        w = W.uniform_potential(n=2000)
        out = ctx.potential_host(w["theta"], w["xs"], w["ys"], w["vs"], w["xt"], w["yt"])
        assert np.isfinite(out).all()
    finally:
        ctx.close()


@pytest.mark.parametrize("bs", (16, 64))
def test_blocksize_matches_reference_build(bs):
    """Block sides other than 32 (the reference's build-time mrag-blocksize) against the
    reference driver built with that BLOCKSIZE."""
    import oracle as O
    g = 2048 // (bs * 32) if bs <= 64 else 1
    w = W.lamb_oseen_force(n=30000, blocks_per_side=max(g, 1), h=1.0 / (bs * max(g, 1)))
    ctx = T.Context(device=0)
    try:
        ctx.set_blocksize(bs)
        xo, yo = ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"],
                                     w["hs"])
        assert len(xo) == len(w["x0s"]) * bs * bs
        rx, ry = O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"],
                              mode=f"exact64_b{bs}", blocksize=bs)
        assert rel_l2(np.r_[xo, yo], np.r_[rx, ry]) < 1e-12
    finally:
        ctx.close()


def test_blocksize_8_equals_32_split(force_case):
    """One 32 x 32 block is sixteen 8 x 8 blocks at the same points (the 8-blocks' origins are
    rounded once more, which can move a brick across an acceptance boundary: agreement to the
    treecode's own truncation error, not to the last bit)."""
    w = force_case
    ctx = T.Context(device=0)
    try:
        x32, y32 = ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"],
                                       w["hs"])
        by, bx = np.meshgrid(np.arange(4), np.arange(4), indexing="ij")
        x0 = (w["x0s"][:, None] + (8 * bx.ravel())[None, :] * w["hs"][:, None]).ravel()
        y0 = (w["y0s"][:, None] + (8 * by.ravel())[None, :] * w["hs"][:, None]).ravel()
        h = np.repeat(w["hs"], 16)
        ctx.set_blocksize(8)
        x8, y8 = ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], x0, y0, h)
        # block 16 b + q of side 8 holds the points of brick q of 32-block b
        nb = len(w["x0s"])
        x8 = x8.reshape(nb, 4, 4, 8, 8).transpose(0, 1, 3, 2, 4).reshape(-1)
        y8 = y8.reshape(nb, 4, 4, 8, 8).transpose(0, 1, 3, 2, 4).reshape(-1)
        assert rel_l2(np.r_[x8, y8], np.r_[x32, y32]) < 1e-9
        for bad in (0, 12, 128):
            with pytest.raises(T.TreecodeError, match="block size"):
                ctx.set_blocksize(bad)
    finally:
        ctx.close()
