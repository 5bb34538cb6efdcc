"""CPU tests of the serving stream driver (2d-treecodes_b200/serving.py) against a stand-in
server: the stream's composition, the open-loop replay, the follow-up advection, and the client
sessions (a resident client is released once, after its last step completes; one-off requests
run on client 0 and are never released)."""
import threading
import time

import numpy as np

import serving as S


class FakeServer:
    """Records what the driver asks of a request server.  `wait_any` completes the newest
    outstanding request whose client has no earlier one outstanding (one client's steps stay in
    order, as on the real server), so the driver must cope with completions out of submission
    order."""

    def __init__(self):
        self.lock = threading.Lock()
        self.submitted = []      # (ticket, kind, client, nsources)
        self.completed = set()
        self.released = []       # (client, tickets completed at the time)
        self.inputs = {}
        self.order = []          # tickets in the order wait_any completed them

    def _submit(self, kind, client, xs, ys, vs):
        with self.lock:
            t = len(self.submitted)
            self.submitted.append((t, kind, client, len(xs)))
            self.inputs[t] = (np.array(xs), np.array(ys), np.array(vs))
            return t

    def submit_potential(self, theta, xs, ys, vs, xt, yt, precision=0, client=0):
        assert len(xt) == len(xs) and np.array_equal(xt, xs) and np.array_equal(yt, ys)
        return self._submit("potential", client, xs, ys, vs)

    def submit_force(self, theta, xs, ys, vs, x0s, y0s, hs, precision=0, client=0):
        assert len(x0s) == len(y0s) == len(hs) >= 1
        return self._submit("force", client, xs, ys, vs)

    def wait(self, ticket):
        with self.lock:
            self.completed.add(ticket)
        return (np.zeros(1),), {"status": 0, "slot": 0, "queue_ms": 0.0, "service_ms": 0.1,
                                "finished_s": time.perf_counter()}

    def wait_any(self):
        with self.lock:
            out = [(t, c) for t, _, c, _ in self.submitted if t not in self.completed]
            assert out, "wait_any with nothing outstanding"
            first = {}
            for t, c in out:
                first.setdefault(c, t)
            ready = [t for t, c in out if c == 0 or first[c] == t]
            t = max(ready)
            self.completed.add(t)
            self.order.append(t)
        return t, (np.zeros(1),), {"status": 0, "slot": 0, "queue_ms": 0.0, "service_ms": 0.1,
                                   "finished_s": time.perf_counter()}

    def release_client(self, client):
        with self.lock:
            self.released.append((client, set(self.completed)))

    def stats(self):
        return {}


def small_stream(nreq, seed):
    return S.make_stream(nreq=nreq, rate_hz=20000.0, seed=seed, log2_min=8, log2_max=12)


def test_stream_composition():
    specs = small_stream(2000, 5)
    assert all(b["t"] >= a["t"] for a, b in zip(specs, specs[1:]))
    force = np.mean([s["kind"] == "force" for s in specs])
    follow = np.mean([s["followup"] for s in specs])
    assert 0.6 < force < 0.8 and 0.15 < follow < 0.25
    ns = np.log2([s["n"] for s in specs if not s["followup"]])
    assert ns.min() >= 8 and ns.max() <= 12
    for s in specs:
        assert s["theta"] in S.THETAS and s["dist"] in S.DISTRIBUTIONS
        assert s["resident"] == (s["last_step"] > 0)
    # a client's steps keep its kind and size, and count up from 0
    by_client = {}
    for s in specs:
        by_client.setdefault(s["client"], []).append(s)
    for steps in by_client.values():
        assert [s["step"] for s in steps] == list(range(len(steps)))
        assert len({(s["kind"], s["n"], s["dist"]) for s in steps}) == 1


def test_clients_released_once_after_their_last_step():
    specs = small_stream(300, 7)
    m = S.Materialiser(log2_max=12, seed=3)
    srv = FakeServer()
    summary, _ = S.run_stream(srv, specs, 1, m)
    assert summary["requests"] == len(specs) and len(srv.completed) == len(specs)
    resident = {s["client"] for s in specs if s["resident"]}
    assert resident, "the stream should have clients with follow-ups"
    released = [c for c, _ in srv.released]
    assert sorted(released) == sorted(resident)          # each exactly once, none else
    assert 0 not in released
    last_ticket = {}
    for (t, _, client, _), s in zip(srv.submitted, specs):
        assert client == (s["client"] if s["resident"] else 0)
        if s["resident"]:
            last_ticket[s["client"]] = t
    for client, done in srv.released:
        assert last_ticket[client] in done                 # after its last step completed


def test_results_collected_in_completion_order():
    specs = small_stream(300, 13)
    m = S.Materialiser(log2_max=12, seed=3)
    srv = FakeServer()
    summary, outs = S.run_stream(srv, specs, 1, m, keep_outputs=True)
    assert sorted(srv.order) == list(range(len(specs)))   # every request exactly once
    assert all(o is not None for o in outs)
    assert summary["p50_ms"] >= 0 and np.isfinite(summary["p99_ms"])


def test_followups_advect_the_previous_step():
    specs = small_stream(300, 11)
    m = S.Materialiser(log2_max=12, seed=3)
    srv = FakeServer()
    S.run_stream(srv, specs, 0, m)
    prev = {}
    for (t, _, _, n), s in zip(srv.submitted, specs):
        xs, ys, vs = srv.inputs[t]
        assert len(xs) == s["n"] == n
        if s["followup"]:
            px, py, pv = prev[s["client"]]
            dx, dy = xs - px, ys - py
            assert np.array_equal(vs, pv)
            assert 0 < np.abs(dx).max() < 1e-2 and 0 < np.abs(dy).max() < 1e-2
        prev[s["client"]] = (xs, ys, vs)
