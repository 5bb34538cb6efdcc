"""Generates the golden fixtures of tests/golden/ from the CPU oracle.

The reference ships no golden vectors, so the fixtures are outputs of the reference itself:
its C++ drivers compiled verbatim (oracle/Makefile) with the restated ISPC kernels, in both
kernel modes (exact64: double constants and logs; faithful: the m4 literals as ISPC floats and
the single-precision log of potential_p2p).  Each fixture holds the seeded inputs, the Morton
keys and sorted sources, the tree in canonical breadth-first order and the outputs.

Run from the repository root after `make -C oracle`:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "2d-treecodes_b200")]

import oracle as O  # noqa: E402
import workloads as W  # noqa: E402


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def cases():
    """name -> workload dict (small seeded inputs covering the reference's code paths)."""
    c = {}
    c["potential_uniform"] = W.uniform_potential(n=3000, seed=11)
    w = W.uniform_potential(n=2500, seed=12)
    # a cluster of 700 coincident sources: one key holds more than a leaf (512) -> level-15 leaf
    w["xs"][:700] = 0.3125
    w["ys"][:700] = 0.6875
    w["xt"], w["yt"] = w["xs"].copy(), w["ys"].copy()
    w["name"] = "potential_coincident_cluster"
    c["potential_coincident_cluster"] = w
    # all coordinates negative: the bounding box's initial maximum of 0 enters the extent
    w = W.uniform_potential(n=2000, seed=13)
    w["xs"] = -1.0 - w["xs"]
    w["ys"] = -3.0 - 2.0 * w["ys"]
    w["xt"], w["yt"] = w["xs"].copy() * 0.999, w["ys"].copy() * 1.001
    w["name"] = "potential_negative_coordinates"
    c["potential_negative_coordinates"] = w
    c["force_lamb_oseen"] = W.lamb_oseen_force(n=6000, blocks_per_side=2, h=1.0 / 64, seed=14)
    # negligible weights: sources far from the vortex carry ~1e-30, so whole quadrants fall
    # below the 1.1e-16 threshold (the all-four and three-of-four cases of upward.cpp:161-214)
    w = W.lamb_oseen_force(n=5000, blocks_per_side=2, h=1.0 / 64, seed=15)
    r = rng(15)
    far = r.random(5000) < 0.3
    w["xs"][far] = 0.02 + 0.2 * r.random(far.sum())
    w["ys"][far] = 0.02 + 0.2 * r.random(far.sum())
    w["vs"][far] = 1e-30 * r.random(far.sum())
    w["name"] = "force_negligible_quadrants"
    c["force_negligible_quadrants"] = w
    # exact zeros among the values: small outlying leaves whose sources all carry zero use the
    # cell centre as com (upward.cpp:71-72), and leaves whose first source in a 4-lane group is
    # zero measure part of their radius about the origin (upward-common.ispc:44-56).  Every
    # inner cell holds > 192 sources, so no cell has zero total weight (which would give 0/0).
    w = W.lamb_oseen_force(n=4000, blocks_per_side=1, h=1.0 / 32, seed=16)
    w["vs"][rng(16).random(4000) < 0.3] = 0.0
    w["name"] = "force_zero_values"
    c["force_zero_values"] = w
    return c


def canonical_arrays(t):
    cn = O.canonical(t)
    return {f"tree_{k}": cn[k] for k in ("level", "cx", "cy", "s", "e", "inner", "mass", "xcom",
                                          "ycom", "r", "exps")}


def make(name, w):
    kind = w["kind"]
    out = {k: w[k] for k in w if isinstance(w[k], np.ndarray)}
    out["theta"] = np.float64(w["theta"])
    keys, xs, ys, vs, bbox = O.sort_sources(w["xs"], w["ys"], w["vs"], kind, "exact64")
    out.update(keys=keys, sorted_x=xs, sorted_y=ys, sorted_v=vs, frame=bbox)
    out.update(canonical_arrays(O.tree(w["xs"], w["ys"], w["vs"], kind, "exact64")))
    for mode in ("exact64", "faithful"):
        if kind == "potential":
            out[f"potential_{mode}"] = O.potential(w["theta"], w["xs"], w["ys"], w["vs"], w["xt"],
                                                   w["yt"], mode)
        else:
            xo, yo = O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"],
                                  w["hs"], mode)
            out[f"xforce_{mode}"] = xo
            out[f"yforce_{mode}"] = yo
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, kind=np.array(kind), **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    for name, w in cases().items():
        make(name, w)
