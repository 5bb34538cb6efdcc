"""One force_mrag problem split by blocks (sharding.py): the shards, solved one after another on
one GPU as separate ranks would solve them, assemble to the unsplit solve bit for bit (the
tree is the same deterministic tree on every rank, and a block's result depends only on it)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "2d-treecodes_b200"))

import sharding            # noqa: E402
import treecodes as T      # noqa: E402
import workloads as W      # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_shards_assemble_to_the_whole_solve(precision):
    w = W.lamb_oseen_force(n=200000, blocks_per_side=6, h=1.0 / 192)
    ctx = T.Context(device=0, precision=precision)
    try:
        xo, yo = ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"],
                                     w["hs"])
        for world in (2, 5):
            parts = [sharding.solve_shard(ctx, w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"],
                                          w["y0s"], w["hs"], r, world) for r in range(world)]
            sx, sy = sharding.assemble(parts, len(w["x0s"]))
            assert np.array_equal(sx, xo) and np.array_equal(sy, yo)
    finally:
        ctx.close()
