"""The library's bounded device waits and capacities, made to run out on purpose.

Every look-back wait in a kernel reads another CTA's published state a bounded number of times
and then raises a device error flag instead of waiting on; traversal stacks stop at their
capacity.  These tests make each of them give up (a look-back tile that never publishes its
state, a tiny stack), check the status the call reports, and check that the next solve on the
same context is correct.  Nothing here faults, traps or hangs the GPU: every wait ends after a
few hundred reads and every access stays in bounds."""
import numpy as np
import pytest

import treecodes as T
import workloads as W
from tc_helpers import gpu_force, gpu_potential

pytestmark = pytest.mark.gpu

TC_ERR_CAPACITY, TC_ERR_TIMEOUT = 3, 4
TC_STALL_SORT, TC_STALL_TREE = 1, 2


@pytest.fixture()
def ctx():
    c = T.Context(device=0)
    yield c
    c.close()


def force_case():
    return W.lamb_oseen_force(n=100000, blocks_per_side=2, h=1.0 / 64, seed=41)


def potential_case():
    return W.uniform_potential(n=50000, seed=42)


def expect_status(fn, status):
    with pytest.raises(T.TreecodeError):
        fn()
    assert T.last_status() == status, T.last_error()


@pytest.mark.parametrize("stall", [TC_STALL_SORT, TC_STALL_TREE])
def test_lookback_wait_runs_out(ctx, stall):
    wf, wp = force_case(), potential_case()
    fresh = T.Context(device=0)
    try:
        ref_f = gpu_force(fresh, wf)
        ref_p = gpu_potential(fresh, wp)
    finally:
        fresh.close()
    ctx.set_wait_test(stall=stall, spin_limit=256)
    expect_status(lambda: gpu_force(ctx, wf), TC_ERR_TIMEOUT)
    assert "bounded device wait" in T.last_error()
    expect_status(lambda: gpu_potential(ctx, wp), TC_ERR_TIMEOUT)
    # the host entry points report the same status and leave nothing in flight
    with pytest.raises(T.TreecodeError):
        ctx.force_mrag_host(wf["theta"], wf["xs"], wf["ys"], wf["vs"], wf["x0s"], wf["y0s"],
                            wf["hs"])
    assert T.last_status() == TC_ERR_TIMEOUT
    ctx.set_wait_test()
    xo, yo = gpu_force(ctx, wf)
    assert np.array_equal(xo, ref_f[0]) and np.array_equal(yo, ref_f[1])
    assert np.array_equal(gpu_potential(ctx, wp), ref_p)


def test_lowered_spin_limit_alone_is_harmless(ctx):
    """A low bound without a stalled tile still completes (waits that make progress do not
    count against it) and gives the same bits."""
    wf = force_case()
    ref = gpu_force(ctx, wf)
    ctx.set_wait_test(spin_limit=1 << 16)
    try:
        got = gpu_force(ctx, wf)
    finally:
        ctx.set_wait_test()
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


def test_traversal_stack_capacity(ctx):
    wf = force_case()
    ref = gpu_force(ctx, wf)
    ctx.set_wait_test(stack_limit=8)
    expect_status(lambda: gpu_force(ctx, wf), TC_ERR_CAPACITY)
    assert "stack" in T.last_error()
    ctx.set_wait_test()
    got = gpu_force(ctx, wf)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


def test_invalid_wait_test_setting(ctx):
    with pytest.raises(T.TreecodeError):
        ctx.set_wait_test(stall=7)
    assert T.last_status() == 1
