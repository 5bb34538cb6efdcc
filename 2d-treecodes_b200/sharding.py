"""One treecode problem split over ranks: force_mrag by blocks, potential by targets.

The blocks of a force_mrag solve are independent, and so are the targets of a potential solve
(drivers/treecode-force.cpp:219-225 and drivers/treecode-potential.cpp:101-102 of the reference
loop over them with no dependence between iterations): every output element has one owner, so
ranks need no exchange while they evaluate.  Each rank builds the whole tree from all the
sources (the tree is replicated) and evaluates a contiguous run of the blocks, or targets, in
Morton order of their positions, so that a rank's share is close together and touches a compact
part of the tree.  Gathering the shards is needed only by a caller that wants every output on
one rank.
"""
from __future__ import annotations

import numpy as np

import treecodes as T


def _spread(v):
    v = (v | (v << 8)) & 0x00FF00FF
    v = (v | (v << 4)) & 0x0F0F0F0F
    v = (v | (v << 2)) & 0x33333333
    return (v | (v << 1)) & 0x55555555


def morton_order(x, y):
    """Indices of the points (x, y) in Morton order (15 bits per axis over their bounding
    square; ties keep index order)."""
    x0s = np.asarray(x, dtype=np.float64)
    y0s = np.asarray(y, dtype=np.float64)
    if len(x0s) == 0:
        return np.zeros(0, dtype=np.int64)
    lo_x, lo_y = x0s.min(), y0s.min()
    ext = max(x0s.max() - lo_x, y0s.max() - lo_y)
    scale = (32767.0 / ext) if ext > 0 else 0.0
    qx = np.clip(((x0s - lo_x) * scale).astype(np.int64), 0, 32767)
    qy = np.clip(((y0s - lo_y) * scale).astype(np.int64), 0, 32767)
    keys = _spread(qx) | (_spread(qy) << 1)
    return np.argsort(keys, kind="stable")


def block_order(x0s, y0s):
    """Block indices in Morton order of their origins."""
    return morton_order(x0s, y0s)


def _run(order, rank, world):
    """The rank-th of `world` near-equal contiguous runs of `order`."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    bounds = np.linspace(0, len(order), world + 1).round().astype(np.int64)
    return order[bounds[rank]:bounds[rank + 1]]


def block_shard(x0s, y0s, rank, world):
    """The blocks rank `rank` of `world` evaluates: the rank-th of `world` near-equal contiguous
    runs of the Morton order (every block in exactly one shard)."""
    return _run(block_order(x0s, y0s), rank, world)


def target_shard(xt, yt, rank, world):
    """The targets rank `rank` of `world` evaluates in a potential solve: the rank-th of
    `world` near-equal contiguous runs of the targets' Morton order."""
    return _run(morton_order(xt, yt), rank, world)


def solve_shard(ctx, theta, xs, ys, vs, x0s, y0s, hs, rank, world, blocksize=T.BLOCKSIZE):
    """This rank's part of a force_mrag solve on `ctx`: (block indices, xout, yout), the outputs
    in the reference's layout over the shard's blocks."""
    idx = block_shard(x0s, y0s, rank, world)
    x0s, y0s, hs = (np.asarray(a, dtype=np.float64)[idx] for a in (x0s, y0s, hs))
    xo, yo = ctx.force_mrag_host(theta, xs, ys, vs, x0s, y0s, hs)
    return idx, xo, yo


def assemble(parts, nblocks, blocksize=T.BLOCKSIZE):
    """Full outputs from every rank's (block indices, xout, yout)."""
    b2 = blocksize * blocksize
    xo = np.empty(nblocks * b2)
    yo = np.empty(nblocks * b2)
    seen = np.zeros(nblocks, dtype=bool)
    for idx, px, py in parts:
        idx = np.asarray(idx)
        if seen[idx].any():
            raise ValueError("a block is owned by two shards")
        seen[idx] = True
        dst = (idx[:, None] * b2 + np.arange(b2)[None, :]).ravel()
        xo[dst] = px
        yo[dst] = py
    if not seen.all():
        raise ValueError("a block is owned by no shard")
    return xo, yo


def solve_potential_shard(ctx, theta, xs, ys, vs, xt, yt, rank, world):
    """This rank's part of a potential solve on `ctx`: (target indices, potentials there)."""
    idx = target_shard(xt, yt, rank, world)
    xt, yt = (np.asarray(a, dtype=np.float64)[idx] for a in (xt, yt))
    return idx, ctx.potential_host(theta, xs, ys, vs, xt, yt)


def assemble_potential(parts, ntargets):
    """Full potential output from every rank's (target indices, values)."""
    out = np.empty(ntargets)
    seen = np.zeros(ntargets, dtype=bool)
    for idx, vals in parts:
        idx = np.asarray(idx)
        if seen[idx].any():
            raise ValueError("a target is owned by two shards")
        seen[idx] = True
        out[idx] = vals
    if not seen.all():
        raise ValueError("a target is owned by no shard")
    return out
