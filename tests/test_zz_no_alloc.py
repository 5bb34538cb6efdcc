"""GPU test of tc_sort_sources_noalloc, the allocation-free source sort.

Callers that cannot allocate device memory (solvers that own every byte through their own
pool, latency-critical loops, services that must not grow their footprint) use this entry
point; its scratch is a fixed static device array shared by all calls.  The test calls it
through the C ABI twice in a row -- a larger input, then a smaller one, so the second call
runs on scratch that still holds the first call's contents -- and compares every output with
the allocating path (tc_tree_build_device) bit for bit, the tolerance the parity tests use
for keys, permutations and sorted sources.  It also checks the size limit.  It creates its
own context, so it passes alone in a fresh process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

import treecodes as T
import workloads as W

pytestmark = pytest.mark.gpu


def noalloc_sort(w):
    import torch
    n = len(w["xs"])
    x, y, v = (torch.as_tensor(w[k]).cuda() for k in ("xs", "ys", "vs"))
    keys = torch.empty(n, dtype=torch.int32, device="cuda")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    xs, ys, vs = (torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(3))
    frame = torch.empty(4, dtype=torch.float64, device="cuda")
    rc = T.load().tc_sort_sources_noalloc(x.data_ptr(), y.data_ptr(), v.data_ptr(), n,
                                          keys.data_ptr(), perm.data_ptr(), xs.data_ptr(),
                                          ys.data_ptr(), vs.data_ptr(), frame.data_ptr(), None)
    assert rc == 0, T.last_error()
    return {k: t.cpu().numpy() for k, t in
            dict(keys=keys, perm=perm, xs=xs, ys=ys, vs=vs, frame=frame).items()}


def test_noalloc_sort_matches_allocating_path_twice():
    import torch
    ctx = T.Context(device=0)
    try:
        for w in (W.vortex_sheet_force(n=1 << 20, blocks_per_side=2, seed=41),
                  W.uniform_potential(n=70001, seed=42)):
            got = noalloc_sort(w)
            ref = ctx.tree("force", *(torch.as_tensor(w[k]).cuda() for k in ("xs", "ys", "vs")))
            for k in ("keys", "perm", "xs", "ys", "vs"):
                assert np.array_equal(got[k], ref[k]), k
            assert np.array_equal(got["frame"][:3], ref["frame"])
            assert np.array_equal(w["xs"][got["perm"]], got["xs"])
    finally:
        ctx.close()


def test_noalloc_sort_rejects_sizes_beyond_its_scratch():
    lib = T.load()
    n = (1 << 20) + 1
    rc = lib.tc_sort_sources_noalloc(None, None, None, n, None, None, None, None, None, None, None)
    assert rc == 1 and T.last_status() == 1       # TC_ERR_INVALID
    assert "1048576" in T.last_error()
