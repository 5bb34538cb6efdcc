"""GPU tests of the serving loop (tc_server_*): a request stream runs with several solves in
flight on separate streams, under a device-memory budget, with resident clients; every result
must equal the same request solved alone on a fresh context (tolerance 0: the kernels are
deterministic, so the mix may not change a single bit)."""
import numpy as np
import pytest

import serving as S
import treecodes as T

pytestmark = pytest.mark.gpu

LOG2_MAX = 16


@pytest.fixture(scope="module")
def materialiser():
    return S.Materialiser(log2_max=LOG2_MAX, seed=77)


def solo(spec, data, precision):
    ctx = T.Context(device=0, precision=precision)
    try:
        if spec["kind"] == "potential":
            return (ctx.potential_host(spec["theta"], data["xs"], data["ys"], data["vs"],
                                       data["xt"], data["yt"]),)
        return ctx.force_mrag_host(spec["theta"], data["xs"], data["ys"], data["vs"],
                                   data["x0s"], data["y0s"], data["hs"])
    finally:
        ctx.close()


def replay_solo(specs, precision):
    m = S.Materialiser(log2_max=LOG2_MAX, seed=77)
    return [solo(s, m(s), precision) for s in specs]


def assert_same(mixed_outs, solo_outs):
    for i, (a, b) in enumerate(zip(mixed_outs, solo_outs)):
        for x, y in zip(a, b):
            assert np.array_equal(x, y), f"request {i}: result differs from the solo solve"


@pytest.mark.parametrize("precision", [0, 1])
def test_stream_results_equal_solo(precision):
    specs = S.make_stream(nreq=48, rate_hz=5000.0, seed=31 + precision, log2_min=10,
                          log2_max=LOG2_MAX, followup_share=0.3)
    m = S.Materialiser(log2_max=LOG2_MAX, seed=77)
    srv = T.Server(slots=4, hbm_budget_bytes=8 << 30, device=0)
    try:
        summary, outs = S.run_stream(srv, specs, precision, m, keep_outputs=True)
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(specs) and st["failed"] == 0
    assert st["max_in_service"] > 1, "no two solves were ever in service together"
    assert any(s["followup"] for s in specs)
    assert_same(outs, replay_solo(specs, precision))
    assert summary["p99_ms"] >= summary["p50_ms"] > 0


def test_wait_any_collects_each_request_once_in_completion_order():
    """tc_server_wait_any: every ticket exactly once, completion stamps (CLOCK_MONOTONIC, the
    clock of time.perf_counter) non-decreasing and within the call, each result equal to the
    request solved alone; with nothing outstanding it reports so at once."""
    import time
    specs = S.make_stream(nreq=24, rate_hz=5000.0, seed=57, log2_min=10, log2_max=LOG2_MAX,
                          followup_share=0.0)
    m = S.Materialiser(log2_max=LOG2_MAX, seed=77)
    datas = [m(s) for s in specs]
    srv = T.Server(slots=4, hbm_budget_bytes=8 << 30, device=0)
    try:
        t0 = time.perf_counter()
        tickets = [S.submit(srv, s, d, 1) for s, d in zip(specs, datas)]
        got, stamps = {}, []
        for _ in tickets:
            t, outs, res = srv.wait_any()
            assert t in tickets and t not in got
            got[t] = outs
            stamps.append(res["finished_s"])
        t1 = time.perf_counter()
        with pytest.raises(T.TreecodeError, match="no request outstanding"):
            srv.wait_any()
    finally:
        srv.close()
    assert stamps == sorted(stamps) and t0 <= stamps[0] and stamps[-1] <= t1
    assert_same([got[t] for t in tickets], [solo(s, d, 1) for s, d in zip(specs, datas)])


def test_budget_limits_concurrency_and_evicts():
    specs = S.make_stream(nreq=24, rate_hz=5000.0, seed=41, log2_min=14, log2_max=LOG2_MAX,
                          followup_share=0.4)
    biggest = max(T.request_footprint(1 if s["kind"] == "force" else 0, s["n"],
                                      s["n"], max(1, round((s["n"] / 2048) ** 0.5)) ** 2, 1)
                  for s in specs)
    budget = int(biggest * 1.6)
    m = S.Materialiser(log2_max=LOG2_MAX, seed=77)
    srv = T.Server(slots=4, hbm_budget_bytes=budget, device=0)
    try:
        _, outs = S.run_stream(srv, specs, 1, m, keep_outputs=True)
        st = srv.stats()
    finally:
        srv.close()
    assert st["failed"] == 0
    assert st["hbm_peak"] <= budget
    assert st["max_in_service"] <= 4
    assert_same(outs, replay_solo(specs, 1))


def test_oversize_request_fails_cleanly(materialiser):
    spec = dict(kind="force", n=1 << 14, dist="uniform", theta=0.5, off=0, followup=False,
                step=0, client=1, noise_off=0, last_step=0, resident=False, t=0.0)
    data = materialiser(spec)
    srv = T.Server(slots=2, hbm_budget_bytes=1 << 20, device=0)
    try:
        t = S.submit(srv, spec, data, 0)
        with pytest.raises(T.TreecodeError, match="status 3"):
            srv.wait(t)
        # the server keeps serving requests that fit
        srv2 = T.Server(slots=1, hbm_budget_bytes=4 << 30, device=0)
        try:
            t2 = S.submit(srv2, spec, data, 0)
            outs, res = srv2.wait(t2)
            assert res["status"] == 0
            assert_same([outs], [solo(spec, data, 0)])
        finally:
            srv2.close()
    finally:
        srv.close()


def test_resident_client_steps_in_order_and_release(materialiser):
    base = dict(kind="potential", n=5000, dist="gaussian_mixture", theta=0.5, off=123,
                followup=False, step=0, client=9, noise_off=0, last_step=3, resident=True,
                t=0.0)
    steps = [dict(base, step=k, followup=k > 0, noise_off=1000 * k) for k in range(4)]
    m = S.Materialiser(log2_max=LOG2_MAX, seed=77)
    datas = [m(s) for s in steps]
    srv = T.Server(slots=3, hbm_budget_bytes=4 << 30, device=0)
    try:
        tickets = [S.submit(srv, s, d, 1) for s, d in zip(steps, datas)]
        outs = [srv.wait(t)[0] for t in tickets]
        st = srv.stats()
        assert st["resident_clients"] == 1
        srv.release_client(9)
        assert srv.stats()["resident_clients"] == 0
    finally:
        srv.close()
    assert_same(outs, [solo(s, d, 1) for s, d in zip(steps, datas)])
    # the steps differ (each advects the previous one), so order mattered
    assert not np.array_equal(outs[0][0], outs[1][0])


def test_sleeping_host_waits_give_the_same_results():
    """tc_set_host_waits(1), the way the server's slots wait, changes only how the host thread
    waits: both solves equal the spinning default bit for bit; other modes are refused."""
    import workloads as W
    w = W.lamb_oseen_force(n=40000, blocks_per_side=2, h=1.0 / 64)
    p = W.uniform_potential(n=30000)
    out = {}
    for mode in (0, 1):
        ctx = T.Context(device=0)
        try:
            ctx.set_host_waits(mode)
            f = ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"],
                                    w["hs"])
            q = ctx.potential_host(p["theta"], p["xs"], p["ys"], p["vs"], p["xt"], p["yt"])
            out[mode] = (f[0], f[1], q)
            for bad in (-1, 2):
                with pytest.raises(T.TreecodeError, match="wait mode"):
                    ctx.set_host_waits(bad)
        finally:
            ctx.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_trimmed_memory_stays_cached_until_released():
    """tc_context_trim frees a context's buffers into the device's pool, which keeps them for
    the next allocations while contexts live; tc_release_cached_memory hands them back."""
    import torch
    import workloads as W
    w = W.lamb_oseen_force(n=1 << 20, blocks_per_side=4, h=1.0 / 128)
    keep = T.Context(device=0)   # another live context: trims and destroys keep the cache
    ctx = T.Context(device=0)
    try:
        ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"])
        held = ctx.device_bytes()
        assert held > 64 << 20
        ctx.trim()
        assert ctx.device_bytes() < 1 << 20
        free0 = torch.cuda.mem_get_info(0)[0]
        T.release_cached_memory(0)
        free1 = torch.cuda.mem_get_info(0)[0]
        assert free1 - free0 > held // 2, (free0, free1, held)
        # the context solves again after the trim, with the same result
        a = ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"],
                                w["hs"])
        b = keep.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"],
                                 w["hs"])
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    finally:
        ctx.close()
        keep.close()


def test_reserved_memory_serves_later_solves():
    """tc_reserve_cached_memory maps memory into the device pool ahead of the solves: device
    free memory drops by about the amount, a solve afterwards is carved from it (free memory
    does not drop again), and tc_release_cached_memory hands the unused part back."""
    import torch
    import workloads as W
    w = W.lamb_oseen_force(n=1 << 20, blocks_per_side=4, h=1.0 / 128)
    free = lambda: torch.cuda.mem_get_info(0)[0]
    keep = T.Context(device=0)   # a live context: the pool keeps what is freed into it
    ctx = T.Context(device=0)
    try:
        T.release_cached_memory(0)
        f0 = free()
        T.reserve_cached_memory(2 << 30, 0)
        f1 = free()
        assert f0 - f1 >= (2 << 30) * 9 // 10, (f0, f1)
        ctx.force_mrag_host(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"])
        assert 0 < ctx.device_bytes() < 1 << 30
        f2 = free()
        assert f1 - f2 < 64 << 20, (f1, f2, ctx.device_bytes())
        T.release_cached_memory(0)
        assert free() - f2 >= 1 << 30
    finally:
        ctx.close()
        keep.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_concurrent_contexts_equal_solo(precision):
    """Four threads, each with its own context, solve half-million-source force problems at
    once, repeatedly: every result equals the problem solved alone, bit for bit.  Each solve
    runs work on two streams of its context, so this exercises the ordering between them under
    load from the other contexts."""
    import threading
    import workloads as W
    ws = [W.lamb_oseen_force(n=1 << 19, blocks_per_side=8, h=1.0 / 256, seed=50 + i)
          for i in range(4)]
    args = [(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"]) for w in ws]
    refs = []
    for a in args:
        ctx = T.Context(device=0, precision=precision)
        try:
            refs.append(ctx.force_mrag_host(*a))
        finally:
            ctx.close()
    results = [None] * len(args)
    errors = []

    def run(i):
        try:
            ctx = T.Context(device=0, precision=precision)
            try:
                results[i] = [ctx.force_mrag_host(*args[i]) for _ in range(4)]
            finally:
                ctx.close()
        except Exception as exc:   # reported below, on the test's thread
            errors.append((i, exc))

    threads = [threading.Thread(target=run, args=(i,)) for i in range(len(args))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for i, outs in enumerate(results):
        for xo, yo in outs:
            assert np.array_equal(xo, refs[i][0]) and np.array_equal(yo, refs[i][1]), i
