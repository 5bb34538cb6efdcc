"""The serving stream: seeded request streams for the request server and an open-loop driver.

A stream is a list of requests with Poisson arrival times.  Each request is a potential or a
force_mrag solve (70% force) with a source count drawn log-uniformly in [2^12, 2^22], sources
drawn from one of the four benchmark distributions (uniform, Gaussian mixture, Lamb-Oseen
vortex, vortex sheet) and theta from {0.3, 0.5, 0.7}.  A fifth of the requests are follow-up
steps of an earlier client: that client's previous sources advected by 1e-3 N(0,1), solved on
the client's resident context, which the driver releases once the client's last step is done.
Potential targets are a copy of the source coordinates; force
targets are a g x g grid of 32 x 32-point blocks tiling [0,1)^2 with g = round(sqrt(N / 2048))
(about N/2 targets).

Source sets are slices of one pre-drawn master set per distribution (2^22 i.i.d. points each),
passed as views, so materialising a request costs no copy and no random draw (a value scaling
for the 1/N-normalised distributions and, for follow-ups, the advection: two O(N) passes over a
slice of a pre-drawn normal array).  The driver replays arrivals open-loop from one thread
(submission) while another collects completions; a request's latency runs from its scheduled
arrival to its completion, so a submitter that falls behind shows up as latency.
"""
from __future__ import annotations

import gc
import math
import threading
import time

import numpy as np

import treecodes as T
import workloads as W

DISTRIBUTIONS = ("uniform", "gaussian_mixture", "lamb_oseen", "vortex_sheet")
THETAS = (0.3, 0.5, 0.7)


def pinned_empty(n):
    """A float64 host array in page-locked memory (torch's pinned allocator), so that the
    library's host-to-device copies of it are direct DMA; plain memory without torch."""
    try:
        import torch
        return torch.empty(int(n), dtype=torch.float64, pin_memory=True).numpy()
    except Exception:   # no CUDA driver: pageable memory works too, only slower
        return np.empty(int(n))


def warm_pinned_cache(max_bytes=1 << 25, per_class=32):
    """Fills torch's page-locked block cache: `per_class` blocks of every power-of-two size
    class from 4 KB to `max_bytes`, allocated and released at once.  The cache keeps freed blocks
    by class, so later `pinned_empty` calls reuse them; an empty class instead calls the driver's
    page-locked allocation, which stalls every solve in flight: on the GPU hosts measured, single
    allocations took up to 0.37 s, and the 2000-request stream with 12 blocks per class made
    225 of them, each stall holding more outputs live and so causing the next (p99 0.6-1.2 s)."""
    held, total, b = [], 0, 4096
    try:
        import torch
        while b <= max_bytes:
            for _ in range(per_class):
                held.append(torch.empty(b, dtype=torch.uint8, pin_memory=True))
                total += b
            b *= 2
    except Exception:   # no CUDA driver: pinned_empty hands out pageable memory then
        return 0
    del held
    return total


def pinned_copy(a):
    out = pinned_empty(len(a))
    out[:] = a
    return out


def _masters(log2_max, seed):
    """Per distribution: x, y and an unnormalised value array of 2^log2_max points (pinned)."""
    n = 1 << log2_max
    r = np.random.Generator(np.random.PCG64(seed))
    out = {}
    u = W.uniform_potential(n=n, seed=seed + 1)
    out["uniform"] = (u["xs"], u["ys"], u["vs"], False)
    g = W.gaussian_mixture_potential(n=n, seed=seed + 2)
    out["gaussian_mixture"] = (g["xs"], g["ys"], g["vs"], False)
    lo = W.lamb_oseen_force(n=n, blocks_per_side=1, seed=seed + 3)
    out["lamb_oseen"] = (lo["xs"], lo["ys"], lo["vs"] * n, True)      # value * N
    vs = W.vortex_sheet_force(n=n, blocks_per_side=1, seed=seed + 4)
    out["vortex_sheet"] = (vs["xs"], vs["ys"], vs["vs"] * n, True)
    out = {k: (pinned_copy(a), pinned_copy(b), pinned_copy(c), sc) for k, (a, b, c, sc) in out.items()}
    noise = r.standard_normal(2 * n)
    return out, noise


def make_stream(nreq=2000, rate_hz=200.0, seed=1455, log2_min=12, log2_max=22,
                force_share=0.7, followup_share=0.2, client_window=32):
    """Request specs (dicts) in arrival order; data are materialised by ``Materialiser``."""
    r = np.random.Generator(np.random.PCG64(seed))
    t = np.cumsum(r.exponential(1.0 / rate_hz, nreq))
    specs = []
    opened = []           # client ids in opening order (follow-ups pick among the latest)
    latest = {}           # client id -> its latest spec
    for i in range(nreq):
        if opened and r.random() < followup_share:
            cid = opened[int(r.integers(max(0, len(opened) - client_window), len(opened)))]
            spec = dict(latest[cid])
            spec.update(t=float(t[i]), followup=True, step=latest[cid]["step"] + 1,
                        noise_off=int(r.integers(0, 1 << 20)))
        else:
            n = int(round(2.0 ** r.uniform(log2_min, log2_max)))
            kind = "force" if r.random() < force_share else "potential"
            cid = len(opened) + 1
            opened.append(cid)
            spec = dict(t=float(t[i]), kind=kind, n=n,
                        dist=DISTRIBUTIONS[int(r.integers(0, len(DISTRIBUTIONS)))],
                        theta=float(THETAS[int(r.integers(0, len(THETAS)))]),
                        off=int(r.integers(0, (1 << log2_max) - n + 1)), followup=False,
                        step=0, client=cid, noise_off=0)
        latest[cid] = spec
        specs.append(spec)
    # a client with follow-ups stays resident on the server; one-off requests use client 0
    for s in specs:
        s["last_step"] = latest[s["client"]]["step"]
        s["resident"] = s["last_step"] > 0
    return specs


class Materialiser:
    """Builds request arrays from the master sets; keeps each resident client's latest
    sources so that a follow-up advects them."""

    def __init__(self, log2_max=22, seed=1456):
        self.log2_max = log2_max
        self.masters, noise = _masters(log2_max, seed)
        self.noise = 1e-3 * noise       # the advection step, scaled once
        self.state = {}
        warm_pinned_cache(8 << log2_max)

    def __call__(self, spec):
        n = spec["n"]
        xm, ym, vm, scaled = self.masters[spec["dist"]]
        if spec["followup"] and spec["client"] in self.state:
            xs, ys, vs = self.state[spec["client"]]
            o = spec["noise_off"] % (len(self.noise) - 2 * n)
            # advected sources in page-locked memory (torch's caching host allocator recycles
            # the blocks), so that the server's copies of them are direct DMA
            xs = np.add(xs, self.noise[o:o + n], out=pinned_empty(n))
            ys = np.add(ys, self.noise[o + n:o + 2 * n], out=pinned_empty(n))
        else:
            sl = slice(spec["off"], spec["off"] + n)
            xs, ys = xm[sl], ym[sl]            # read-only views of the master set
            vs = np.divide(vm[sl], n, out=pinned_empty(n)) if scaled else vm[sl]
        if spec["resident"]:
            if spec["step"] >= spec["last_step"]:
                self.state.pop(spec["client"], None)
            else:
                self.state[spec["client"]] = (xs, ys, vs)
        if spec["kind"] == "potential":
            # targets at the source coordinates; the server only reads its host inputs, so the
            # same memory may serve both
            return dict(xs=xs, ys=ys, vs=vs, xt=xs, yt=ys, ntargets=n)
        g = max(1, int(round(math.sqrt(n / 2048.0))))
        x0, y0, hs = W.mrag_grid(g, 1.0 / (32 * g))
        return dict(xs=xs, ys=ys, vs=vs, x0s=x0, y0s=y0, hs=hs, ntargets=g * g * 1024)


def submit(server, spec, data, precision):
    client = spec["client"] if spec["resident"] else 0
    if spec["kind"] == "potential":
        return server.submit_potential(spec["theta"], data["xs"], data["ys"], data["vs"],
                                       data["xt"], data["yt"], precision=precision, client=client)
    return server.submit_force(spec["theta"], data["xs"], data["ys"], data["vs"], data["x0s"],
                               data["y0s"], data["hs"], precision=precision, client=client)


def run_stream(server, specs, precision, materialise, keep_outputs=False):
    """Open-loop replay of `specs` on `server`.  Returns a summary dict (p50/p99 latency from
    scheduled arrival to the server's completion stamp, aggregate Mtargets/s over the stream's
    span) and, if asked, outputs.  Results are collected in completion order
    (`Server.wait_any`), so each request's outputs are released as soon as it is done."""
    index = {}                       # ticket -> (request number, submission time)
    lock = threading.Lock()
    permits = threading.Semaphore(0)   # one per submitted request, one more at the end
    submitted = [None]               # the number submitted, once submission is over
    records = [None] * len(specs)
    outputs = [None] * len(specs) if keep_outputs else None
    errors = []

    def collector():
        collected = 0
        while True:
            permits.acquire()
            with lock:
                if submitted[0] is not None and collected >= submitted[0]:
                    return
            collected += 1
            try:
                ticket, outs, res = server.wait_any()
            except T.TreecodeError as e:
                with lock:
                    i = index.pop(getattr(e, "ticket", None), (None,))[0]
                errors.append((i, str(e)))
                continue
            with lock:
                i, t_sub = index.pop(ticket)
            # the server's completion stamp (CLOCK_MONOTONIC, perf_counter's clock)
            seen = time.perf_counter()
            fin = res["finished_s"]
            t_done = fin if t_sub <= fin <= seen else seen
            records[i] = dict(res, t_done=t_done, t_sub=t_sub)
            spec = specs[i]
            if spec["resident"] and spec["step"] == spec["last_step"]:
                server.release_client(spec["client"])   # the client's session is over
            if keep_outputs:
                outputs[i] = outs

    th = threading.Thread(target=collector)
    # no cyclic garbage collection while the stream runs: a full collection holds the
    # interpreter lock, during which neither the submitting nor the collecting thread runs
    gc.collect()
    gc_was_on = gc.isenabled()
    gc.disable()
    th.start()
    t0 = time.perf_counter()
    count = 0
    try:
        for i, spec in enumerate(specs):
            data = materialise(spec)
            now = time.perf_counter() - t0
            if spec["t"] > now:
                time.sleep(spec["t"] - now)
            t_sub = time.perf_counter()
            with lock:   # the ticket is known to the collector before it can be collected
                ticket = submit(server, spec, data, precision)
                index[ticket] = (i, t_sub)
            count += 1
            permits.release()
    finally:
        with lock:
            submitted[0] = count
        permits.release()
        th.join()
        if gc_was_on:
            gc.enable()
    if errors:
        raise T.TreecodeError(f"{len(errors)} requests failed, first: {errors[0]}")
    lat = np.array([(r["t_done"] - t0) * 1e3 - s["t"] * 1e3 for r, s in zip(records, specs)])
    service = np.array([r["service_ms"] for r in records])
    queue = np.array([r["queue_ms"] for r in records])
    targets = sum(s["n"] if s["kind"] == "potential" else
                  max(1, int(round(math.sqrt(s["n"] / 2048.0)))) ** 2 * 1024 for s in specs)
    span = max(r["t_done"] for r in records) - t0 - specs[0]["t"]
    slow = np.argsort(-lat)[:5]
    summary = dict(requests=len(specs), precision="mixed" if precision else "fp64",
                   p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                   mean_ms=float(lat.mean()), max_ms=float(lat.max()),
                   service_p50_ms=float(np.percentile(service, 50)),
                   queue_p99_ms=float(np.percentile(queue, 99)),
                   mtargets_per_s=targets / span / 1e6, span_s=span,
                   offered_rate_hz=len(specs) / specs[-1]["t"] if specs[-1]["t"] > 0 else None,
                   slowest=[dict(request=int(i), kind=specs[i]["kind"], n=specs[i]["n"],
                                 arrival_s=round(specs[i]["t"], 4), latency_ms=float(lat[i]),
                                 queue_ms=float(queue[i]), service_ms=float(service[i]))
                            for i in slow],
                   server=server.stats())
    return summary, outputs
