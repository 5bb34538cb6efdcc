#!/usr/bin/env python
"""Benchmark of the B200 treecode: one JSON line on stdout (rank 0).

A step is one force_mrag solve (sort, tree, upward pass, interaction lists, far + near field)
of the vortex-sheet workload: 16,777,216 sources on a perturbed sheet, 4096 MRAG blocks of
32 x 32 targets (4,194,304 targets), theta = 0.5, in the mixed-precision form (default) or the
plain FP64 form (--precision fp64).  With the mixed form the line also carries the plain FP64
form measured on the same inputs (`plain_fp64`), so the mixed-vs-FP64 ratio is in one run.

  value     whole-job throughput (Mtargets/s) with inputs resident in HBM, CUDA events on the
            library's stream, max over ranks
  accuracy  relative L2 / max error against the FP64 direct sum on a strided target sample
  e2e       the same metric through the C ABI with pinned host buffers (host->device copies and
            the result read-back timed): tc_force_mrag_host at the run's precision, and the
            reference-compatible treecode_force_mrag (FP64) beside it
  roofline  the evaluation kernels (k_force_far: E2L, L2P, E2P; k_force_near: P2P), each timed
            alone in the library's serialised timing mode: algorithmic flops per launch / its
            event time, against the measured FMA throughput of this GPU (FP64, or FP32 for the
            mixed form); DRAM traffic per launch from the committed ncu captures
  e2e_fp64  the plain FP64 form through the reference-compatible treecode_force_mrag, host
            buffers: the matched-precision figure against the reference arm
  cpu_baseline  the reference's drivers (oracle/_ref) on the host cores: whole calls, measured

--impl reference times the reference's own CPU implementation instead (rank 0 only): one
whole treecode_force_mrag call per step on every host core.
Multi-GPU (torchrun): every rank solves its own independent copy of the workload (weak
scaling, seeds differ by rank); only the timing barrier/max-reduction is collective.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "2d-treecodes_b200"))

import workloads  # noqa: E402

METRIC = "Mtargets/s at stated err vs FP64 direct: mixed vs FP64 GPU; serve p50/p99 ms"
ORDER_FORCE = 24
PHASES = ("sort_ms", "tree_ms", "upward_ms", "lists_ms", "eval_ms", "total_ms", "eval_kernel_ms",
          "far_kernel_ms")
PROFILES = os.path.join(ROOT, "profiles")
L2_BYTES = 126 << 20


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--workload", default="vortex_sheet_force",
                   choices=sorted(workloads.WORKLOADS))
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--accuracy-targets", type=int, default=4096)
    p.add_argument("--single", action="store_true",
                   help="only `warmup` + `steps` device solves and a timing line (for profilers)")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    p.add_argument("--theta", type=float, default=None, help="override the workload's theta")
    p.add_argument("--sources", type=int, default=None,
                   help="override the workload's source count (reduced cases for profilers)")
    p.add_argument("--blocks-per-side", type=int, default=None,
                   help="override a force workload's MRAG grid (h = 1 / (32 x blocks per side))")
    p.add_argument("--serving-requests", type=int, default=2000,
                   help="requests of the serving stream")
    p.add_argument("--serving-rate", type=float, default=200.0, help="Poisson arrival rate, 1/s")
    p.add_argument("--serving-slots", type=int, default=4)
    p.add_argument("--serving-budget-gb", type=float, default=40.0)
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--scaling", choices=["weak", "strong"], default="weak",
                   help="weak: every rank solves its own copy of the workload; strong: the ranks "
                        "split one problem (force blocks / potential targets in Morton order, "
                        "the tree built by every rank)")
    return p.parse_args()


def make_workload(name, seed_offset=0, theta=None, sources=None, blocks_per_side=None):
    fn = workloads.WORKLOADS[name]
    import inspect
    seed = inspect.signature(fn).parameters["seed"].default + seed_offset
    kw = {}
    if sources is not None:
        kw["n"] = sources
    if blocks_per_side is not None:
        kw["blocks_per_side"] = blocks_per_side
    w = fn(seed=seed, **kw)
    if theta is not None:
        w["theta"] = float(theta)
        w["name"] += f"_theta{theta:g}"
    return w


def n_targets(w):
    return len(w["x0s"]) * 1024 if w["kind"] == "force" else len(w["xt"])


# ------------------------------------------------------------------------------- distributed
def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() and args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        # a short timeout: a rank that never arrives ends the others' collective with an error
        dist.init_process_group(backend, timeout=timedelta(seconds=60))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws, device=None):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------- roofline
def algorithmic_flops(stats, kind="force"):
    """Per-solve flops of the evaluation with fixed per-unit weights, by kernel.  force_mrag
    (p=24): far field (k_force_far) E2L 4p^2+20p per (brick, cell), L2P 10p per target, E2P
    16p+8 per (target, cell); near field (k_force_near) P2P 11 per pair (1 division).
    potential (p=12, one kernel, k_potential_eval): P2P 8 per pair (1 log), E2P 10p+8 per
    (target, cell)."""
    if kind == "potential":
        p = 12
        return {"k_potential_eval": 8.0 * stats["p2p_pairs"] + (10 * p + 8) * stats["e2p_pairs"]}
    p = ORDER_FORCE
    return {"k_force_far": (16 * p + 8) * stats["e2p_pairs"] + (4 * p * p + 20 * p) * stats["e2l_pairs"]
            + 10.0 * p * stats["l2p_targets"],
            "k_force_near": 11.0 * stats["p2p_pairs"]}


def read_profile_traffic(kernel, mixed, workload):
    """DRAM bytes per launch of `kernel` (the form that was timed) from the committed ncu
    summary of the same workload (profiles/<kernel>[.mixed].<workload>.txt), or None."""
    name = f"{kernel}{'.mixed' if mixed else ''}.{workload}.txt"
    try:
        with open(os.path.join(PROFILES, name)) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# ------------------------------------------------------------------------------- CPU reference
def _capture_stdout(fn):
    """Runs fn() with file descriptor 1 redirected to a temporary file; returns (result, text).
    The reference's force driver prints per-thread and phase timers on stdout."""
    libc = ctypes.CDLL(None)
    log = tempfile.TemporaryFile(mode="w+b")
    saved = os.dup(1)
    try:
        sys.stdout.flush()
        os.dup2(log.fileno(), 1)
        out = fn()
        libc.fflush(None)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
    log.seek(0)
    text = log.read().decode(errors="replace")
    log.close()
    return out, text


def cpu_reference_step(w, sample_targets=1 << 19):
    """One step of the reference's CPU implementation (oracle/_ref: the reference's drivers
    compiled verbatim + the restated ISPC kernels, node capacity raised for large inputs,
    OpenMP on every host core).  force_mrag: one whole call over all sources and all blocks,
    timed by the wall clock (measured, nothing scaled).  potential (a sample, since a 4M-target
    call takes seconds to tens of seconds): the tree build alone (no targets) and the build
    plus an evenly strided sample of `sample_targets` targets; the difference is scaled to all
    targets.  Returns (seconds for the full workload, description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # the checker / CPU baseline only
    if w["kind"] == "potential":
        m = len(w["xt"])
        stride = max(1, m // sample_targets)
        idx = np.arange(0, m, stride)[:sample_targets]

        def run(ix):
            t0 = time.perf_counter()
            O.potential(w["theta"], w["xs"], w["ys"], w["vs"], w["xt"][ix], w["yt"][ix],
                        mode="big")
            return time.perf_counter() - t0

        build = run(idx[:0])
        sample = run(idx)
        evals = max(sample - build, 0.0)
        full = build + evals * m / len(idx)
        desc = (f"tree build of all {len(w['xs'])} sources ({build:.3f} s, timed alone) + "
                f"evaluation of {len(idx)} of {m} targets (every {stride}th; {evals:.3f} s) "
                f"scaled by {m}/{len(idx)}")
        return full, desc
    nb = len(w["x0s"])

    def run():
        t0 = time.perf_counter()
        O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"], w["y0s"], w["hs"],
                     mode="big")
        return time.perf_counter() - t0

    wall, text = _capture_stdout(run)
    # drivers/treecode-force.cpp:234 prints "UP: <s>s DW: <s>s" (tree build + upward pass,
    # then the evaluation of the blocks); reported beside the measured wall time
    mt = re.findall(r"UP:\s*([0-9.eE+-]+)s\s+DW:\s*([0-9.eE+-]+)s", text)
    split = (f"; the driver's own timers: UP {float(mt[-1][0]):.3f} s, DW {float(mt[-1][1]):.3f} s"
             if mt else "")
    desc = (f"one whole treecode_force_mrag call: tree build + upward pass of all "
            f"{len(w['xs'])} sources and the evaluation of all {nb} blocks, wall time "
            f"{wall:.3f} s (measured, not scaled){split}")
    return wall, desc


def bench_config(w, flush_desc):
    """The `config` object of both arms: the workload alone, identical in both (the arithmetic
    is in each line's `dtype` and `precision`)."""
    return {"workload": w["name"], "theta": w["theta"],
            "order": ORDER_FORCE if w["kind"] == "force" else 12,
            "sources": len(w["xs"]), "targets": n_targets(w), "l2": flush_desc}


def l2_desc(w):
    in_bytes = sum(int(a.nbytes) for a in w.values() if isinstance(a, np.ndarray))
    if in_bytes >= 2 * L2_BYTES:
        return f"inputs larger than L2 ({in_bytes / 1e6:.0f} MB per step)"
    return f"L2 flushed before every timed step (inputs {in_bytes / 1e6:.1f} MB)"


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    w = make_workload(args.workload, theta=args.theta, sources=args.sources,
                      blocks_per_side=args.blocks_per_side)
    cores = os.cpu_count()
    for _ in range(args.warmup):
        cpu_reference_step(w)
    tot = 0.0
    desc = ""
    for _ in range(args.steps):
        t, desc = cpu_reference_step(w)
        tot += t
    ms = tot / args.steps * 1e3
    val = n_targets(w) / (ms * 1e-3) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "Mtargets/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PCG64; the reference's datasets are not available)",
        "precision": "fp64",
        "config": bench_config(w, l2_desc(w)),
        "cpu_baseline": {"value": val, "unit": "Mtargets/s", "cores": cores, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": val, "unit": "Mtargets/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------- GPU arm
def run_b200(args, ws, rank, local):
    import ctypes
    import torch
    import treecodes as T

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA GPU")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    strong = args.scaling == "strong"
    w = make_workload(args.workload, seed_offset=0 if strong else rank, theta=args.theta,
                      sources=args.sources, blocks_per_side=args.blocks_per_side)
    kind = w["kind"]
    # targets of the whole job: every rank's own problem (weak) or the one split problem (strong)
    job_m = n_targets(w) * (1 if strong else ws)
    if strong and ws > 1:
        import sharding
        w = dict(w)
        if kind == "force":
            idx = sharding.block_shard(w["x0s"], w["y0s"], rank, ws)
            for k in ("x0s", "y0s", "hs"):
                w[k] = np.ascontiguousarray(w[k][idx])
        else:
            idx = sharding.target_shard(w["xt"], w["yt"], rank, ws)
            for k in ("xt", "yt"):
                w[k] = np.ascontiguousarray(w[k][idx])
    mixed = args.precision == "mixed"
    ctx = T.Context(device=local, precision=1 if mixed else 0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    d = {k: torch.as_tensor(w[k]).to(dev) for k in w if isinstance(w[k], np.ndarray)}
    m = n_targets(w)
    out = [torch.empty(m, dtype=torch.float64, device=dev) for _ in range(2 if kind == "force" else 1)]

    def solve():
        if kind == "force":
            ctx.force_mrag_device(w["theta"], d["xs"], d["ys"], d["vs"], d["x0s"], d["y0s"],
                                  d["hs"], out[0], out[1])
        else:
            ctx.potential_device(w["theta"], d["xs"], d["ys"], d["vs"], d["xt"], d["yt"], out[0])

    if args.single:
        for _ in range(args.warmup):
            solve()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            solve()
        torch.cuda.synchronize()
        print(json.dumps({"single": w["name"], "precision": args.precision,
                          "ms_per_step": (time.perf_counter() - t0) * 1e3 / max(args.steps, 1),
                          "stats": ctx.stats()}))
        ctx.close()
        return 0

    in_bytes = sum(int(a.nbytes) for a in w.values() if isinstance(a, np.ndarray))
    flush = (torch.zeros((2 * L2_BYTES) // 8, dtype=torch.float64, device=dev)
             if in_bytes < 2 * L2_BYTES else None)

    def timed(precision, steps, sample_clocks=False):
        """Device time per step of `steps` solves (CUDA events on the library's stream, max over
        ranks), after warm-up; returns (ms, kernel launches, clock record)."""
        ctx.set_precision(precision)
        for _ in range(max(args.warmup, 3)):
            solve()
        torch.cuda.synchronize()
        sampler = None
        if sample_clocks:
            sampler = ClockSampler(local)
            sampler.start()
            time.sleep(0.3)
        barrier(ws)
        torch.cuda.synchronize()
        launches = 0
        if flush is None:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                solve()
                launches += ctx.stats()["launches"]
            e1.record(stream)
            torch.cuda.synchronize()
            total = e0.elapsed_time(e1)
        else:
            # inputs smaller than L2: every timed step starts after a write of a buffer twice
            # the L2 size, outside the events
            total = 0.0
            for _ in range(steps):
                with torch.cuda.stream(stream):
                    flush.add_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                solve()
                e1.record(stream)
                launches += ctx.stats()["launches"]
                torch.cuda.synchronize()
                total += e0.elapsed_time(e1)
        barrier(ws)
        clocks = sampler.stop() if sampler else None
        return max_over_ranks(total / steps, ws, dev), launches, clocks

    def phases(precision):
        """Phase times of one solve (events inside the library) and its work counters; then the
        evaluation kernels' times with each kernel alone on the GPU (timing mode 2: the force's
        near and far field one after the other, after the upward pass), for the roofline."""
        ctx.set_precision(precision)
        out_st = None
        for mode in (1, 2):
            ctx.set_timing(mode)
            runs = []
            for _ in range(5):
                solve()
                runs.append(ctx.stats())
            ctx.set_timing(0)
            st = dict(runs[-1])
            for k in PHASES:
                st[k] = statistics.median(r[k] for r in runs)
            if mode == 1:
                out_st = st
            else:
                out_st["isolated_eval_kernel_ms"] = st["eval_kernel_ms"]
                out_st["isolated_far_kernel_ms"] = st["far_kernel_ms"]
        return out_st

    def accuracy(precision):
        """Relative L2 / max error against the FP64 direct sum on a strided target sample."""
        ctx.set_precision(precision)
        solve()
        torch.cuda.synchronize()
        step = max(1, m // args.accuracy_targets)
        idx = torch.arange(7, m, step, device=dev)[: args.accuracy_targets]
        if kind == "force":
            ib, rem = idx // 1024, idx % 1024
            xt = d["x0s"][ib] + (rem % 32).double() * d["hs"][ib]
            yt = d["y0s"][ib] + (rem // 32).double() * d["hs"][ib]
            rx = torch.empty(len(idx), dtype=torch.float64, device=dev)
            ry = torch.empty_like(rx)
            ctx.direct_force_device(d["xs"], d["ys"], d["vs"], xt, yt, rx, ry)
            got, ref = torch.cat([out[0][idx], out[1][idx]]), torch.cat([rx, ry])
        else:
            ref = torch.empty(len(idx), dtype=torch.float64, device=dev)
            ctx.direct_potential_device(d["xs"], d["ys"], d["vs"], d["xt"][idx], d["yt"][idx], ref)
            got = out[0][idx]
        return {"rel_l2_vs_fp64_direct": float((got - ref).norm() / ref.norm()),
                "max_abs_err": float((got - ref).abs().max()), "targets_sampled": int(len(idx))}

    prec = 1 if mixed else 0
    ms, launches, clocks = timed(prec, args.steps, sample_clocks=True)
    value = job_m / (ms * 1e-3) / 1e6
    st = phases(prec)
    acc = accuracy(prec)
    other = None
    if mixed:   # the plain FP64 form on the same inputs, for the mixed-vs-FP64 ratio
        ms64, _, _ = timed(0, args.steps)
        other = {"precision": "fp64", "value": job_m / (ms64 * 1e-3) / 1e6, "unit": "Mtargets/s",
                 "ms_per_step": ms64, "accuracy": accuracy(0),
                 "phase_ms": {k: v for k, v in phases(0).items() if k.endswith("_ms")}}
    ctx.set_precision(prec)

    # ---- dominant kernel: the evaluation launches, timed by events on the library's stream
    # (force: the far-field and near-field kernels separately; the longer one is the headline)
    flops = algorithmic_flops(st, kind)
    peak = T.measure_fma_peak(not mixed)
    # each kernel timed alone on the GPU (in a solve the near field shares the SMs with the
    # upward pass and the far field)
    if kind == "force":
        times = {"k_force_far": st["isolated_far_kernel_ms"],
                 "k_force_near": st["isolated_eval_kernel_ms"] - st["isolated_far_kernel_ms"]}
    else:
        times = {"k_potential_eval": st["isolated_eval_kernel_ms"]}
    wl = w["name"].split("_N")[0]
    kernels = {}
    for kname, kms in times.items():
        ach = flops[kname] / (kms * 1e-3) / 1e12 if kms > 0 else None
        kernels[kname] = {"achieved": ach, "frac": ach / peak if ach else None, "launch_ms": kms,
                          "algorithmic_flops_per_launch": flops[kname],
                          "traffic": read_profile_traffic(kname, mixed, wl)}
    top = max(times, key=times.get)
    tot_flops = sum(flops.values())
    roofline = {"kernel": top, "bound": "fp32" if mixed else "fp64",
                "achieved": kernels[top]["achieved"], "peak": peak, "unit": "TFLOP/s",
                "frac": kernels[top]["frac"], "traffic": kernels[top]["traffic"],
                "peak_source": ("measured %s FMA throughput of this GPU (tc_measure_fma_peak)"
                                % ("FP32" if mixed else "FP64")),
                "algorithmic_flops_per_launch": kernels[top]["algorithmic_flops_per_launch"],
                "launch_ms": kernels[top]["launch_ms"],
                "kernels": kernels,
                "evaluation": {"achieved": tot_flops / (sum(times.values()) * 1e-3) / 1e12,
                               "frac": tot_flops / (sum(times.values()) * 1e-3) / 1e12 / peak,
                               "launch_ms": sum(times.values()),
                               "algorithmic_flops_per_launch": tot_flops,
                               "in_solve_ms": st["eval_kernel_ms"],
                               "note": "launch_ms: the kernels each alone on the GPU; in_solve_ms: "
                                       "their event times inside a solve, where they share the "
                                       "SMs with each other and with the upward pass"},
                "phase_ms": {k: st[k] for k in PHASES}}

    # ---- end to end through the C ABI with pinned host buffers (host -> device copies and the
    # read-back of the results inside the timed region)
    lib = T.load()
    keys = ("xs", "ys", "vs", "x0s", "y0s", "hs") if kind == "force" else ("xs", "ys", "vs", "xt", "yt")
    pin = {k: torch.as_tensor(w[k]).pin_memory() for k in keys}
    hout = [torch.empty(m, dtype=torch.float64).pin_memory() for _ in out]
    P = lambda t: ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))  # noqa: E731
    n = len(w["xs"])

    def solve_host_ctx():   # tc_force_mrag_host / tc_potential_host: the context's precision
        if kind == "force":
            rc = lib.tc_force_mrag_host(ctx.h, w["theta"], P(pin["xs"]), P(pin["ys"]), P(pin["vs"]), n,
                                        P(pin["x0s"]), P(pin["y0s"]), P(pin["hs"]), len(w["x0s"]),
                                        P(hout[0]), P(hout[1]))
        else:
            rc = lib.tc_potential_host(ctx.h, w["theta"], P(pin["xs"]), P(pin["ys"]), P(pin["vs"]), n,
                                       P(pin["xt"]), P(pin["yt"]), m, P(hout[0]))
        if rc != 0:
            raise RuntimeError(lib.treecode_last_error().decode())

    def solve_host_ref():   # the reference-compatible entry points (plain FP64)
        if kind == "force":
            lib.treecode_force_mrag(w["theta"], P(pin["xs"]), P(pin["ys"]), P(pin["vs"]), n,
                                    P(pin["x0s"]), P(pin["y0s"]), P(pin["hs"]), len(w["x0s"]),
                                    P(hout[0]), P(hout[1]))
        else:
            lib.treecode_potential(w["theta"], P(pin["xs"]), P(pin["ys"]), P(pin["vs"]), n,
                                   P(pin["xt"]), P(pin["yt"]), m, P(hout[0]))
        if lib.treecode_last_status() != 0:
            raise RuntimeError(lib.treecode_last_error().decode())

    def wall(fn):
        for _ in range(max(args.warmup, 3)):
            fn()
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            fn()
        t1 = time.perf_counter()
        return max_over_ranks((t1 - t0) / args.steps * 1e3, ws, dev)

    h2d = sum(t.numel() * 8 for t in pin.values())
    d2h = sum(t.numel() * 8 for t in hout)
    e2e_ms = wall(solve_host_ctx)
    e2e_ref_ms = wall(solve_host_ref)
    e2e = {"value": job_m / (e2e_ms * 1e-3) / 1e6, "unit": "Mtargets/s", "ms_per_step": e2e_ms,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "api": ("tc_force_mrag_host" if kind == "force" else "tc_potential_host")
           + " (C ABI, host pointers, %s)" % args.precision,
           "reference_entry_point": {
               "api": ("treecode_force_mrag" if kind == "force" else "treecode_potential")
               + " (C ABI, host pointers, FP64)",
               "value": job_m / (e2e_ref_ms * 1e-3) / 1e6, "ms_per_step": e2e_ref_ms}}

    e2e_fp64 = {"value": job_m / (e2e_ref_ms * 1e-3) / 1e6, "unit": "Mtargets/s",
                "ms_per_step": e2e_ref_ms, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": e2e["reference_entry_point"]["api"],
                "note": "plain FP64 through the reference-compatible entry point: the "
                        "matched-precision figure against the reference arm"}

    # ---- CPU baseline (rank 0, N = 1): one untimed call, then the mean of two measured calls
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cpu_reference_step(w)
            runs = [cpu_reference_step(w) for _ in range(2)]
            t_full = sum(t for t, _ in runs) / len(runs)
            cpu = {"value": m / t_full / 1e6, "unit": "Mtargets/s", "cores": os.cpu_count(),
                   "kind": "reference",
                   "sample": f"mean of 2 calls after 1 untimed; last: {runs[-1][1]}"}
        except Exception as exc:  # the oracle libraries are built in the source container
            cpu = {"value": None, "unit": "Mtargets/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": f"unavailable: {exc}"}

    # ---- serving stream (N = 1): the same stream in the mixed and the plain FP64 form
    serving = None
    if ws == 1 and not args.no_serving and args.serving_requests > 0:
        serving = run_serving(args, T)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mtargets/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None,
            "dtype": "f32+f64" if mixed else "f64",
            "data": "synthetic (seeded PCG64; the reference's datasets are not available)",
            "precision": args.precision,
            "config": bench_config(w, l2_desc(w)),
            "parallelism": (f"{ws} independent solves (one per GPU)" if not strong else
                            f"one problem split over {ws} GPUs (tree built on every GPU)"),
            "accuracy": acc,
            "plain_fp64": other,
            "e2e": e2e,
            "e2e_fp64": e2e_fp64,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches,
            "serving": serving,
        }
        print(json.dumps(line))
    ctx.close()
    return 0


def host_pinned_allocs():
    import torch
    return int(torch.cuda.host_memory_stats().get("num_host_alloc", 0))


def device_free_bytes():
    import torch
    return int(torch.cuda.mem_get_info()[0])


def run_serving(args, T):
    """The serving stream on a request server: p50/p99 latency from arrival and aggregate
    Mtargets/s, mixed and plain FP64 on the same seeded stream.  Inputs and outputs live in
    page-locked host memory; a short stream of other requests warms the server up first."""
    import serving as S
    specs = S.make_stream(nreq=args.serving_requests, rate_hz=args.serving_rate)
    out = {"config": {"requests": len(specs), "rate_hz": args.serving_rate,
                      "slots": args.serving_slots, "hbm_budget_gb": args.serving_budget_gb,
                      "sources": "log-uniform [2^12, 2^22]", "force_share": 0.7,
                      "followup_share": 0.2, "theta": list(S.THETAS),
                      "distributions": list(S.DISTRIBUTIONS), "host_memory": "page-locked",
                      "warm_up": "60 requests of another seed in each form, not counted",
                      "latency": "scheduled arrival to the server's completion stamp "
                                 "(host monotonic clock)"}}
    m = S.Materialiser()
    srv = T.Server(slots=args.serving_slots,
                   hbm_budget_bytes=int(args.serving_budget_gb * (1 << 30)),
                   host_alloc=S.pinned_empty)
    try:
        warm = S.make_stream(nreq=60, rate_hz=args.serving_rate, seed=99)
        for precision in (1, 0):
            m.state.clear()
            S.run_stream(srv, warm, precision, m)
        for precision, name in ((1, "mixed"), (0, "fp64")):
            m.state.clear()
            host0, free0 = host_pinned_allocs(), device_free_bytes()
            summary, _ = S.run_stream(srv, specs, precision, m)
            # stalls outside the solves: page-locked blocks the host allocator had to add, and
            # device memory the stream-ordered pool had to map, during the stream
            summary["host_pinned_allocs"] = host_pinned_allocs() - host0
            summary["device_free_drop_gb"] = (free0 - device_free_bytes()) / 1e9
            out[name] = summary
    finally:
        srv.close()
    return out


def main():
    args = parse_args()
    ws, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            rc = run_reference(args, ws, rank)
        else:
            rc = run_b200(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
