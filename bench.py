#!/usr/bin/env python
"""Benchmark of the B200 treecode: one JSON line on stdout (rank 0).

A step is one treecode_force_mrag solve (sort, tree, upward pass, interaction lists,
far + near field) of the vortex-sheet workload: 16,777,216 sources on a perturbed sheet,
4096 MRAG blocks of 32 x 32 targets (4,194,304 targets), theta = 0.5, plain FP64.

  value     whole-job throughput (Mtargets/s) with inputs resident in HBM, CUDA events on the
            library's stream, max over ranks
  e2e       the same metric through the reference-compatible C entry point treecode_force_mrag
            with pinned host buffers (host->device copies and the result read-back timed)
  roofline  the dominant kernel (k_force_eval): algorithmic FP64 flops per launch / its event
            time, against the measured FP64 FMA throughput of this GPU; DRAM traffic per launch
            from the committed ncu capture
  cpu_baseline  the reference's drivers (oracle/_ref) on the host cores, bounded sample

--impl reference times the reference's own CPU implementation instead (rank 0 only).
Multi-GPU (torchrun): every rank solves its own independent copy of the workload (weak
scaling, seeds differ by rank); only the timing barrier/max-reduction is collective.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "2d-treecodes_b200"))

import workloads  # noqa: E402

METRIC = "Mtargets/s at stated err vs FP64 direct: mixed vs FP64 GPU; serve p50/p99 ms"
ORDER_FORCE = 24
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "k_force_eval.vortex_sheet_force.txt")


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
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    return p.parse_args()


def make_workload(name, seed_offset=0):
    fn = workloads.WORKLOADS[name]
    import inspect
    seed = inspect.signature(fn).parameters["seed"].default + seed_offset
    return fn(seed=seed)


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
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
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
def algorithmic_flops(stats, p=ORDER_FORCE):
    """Per-solve flops of the evaluation kernel with fixed per-unit weights: P2P 11 per pair
    (1 division), E2P 16p+8 per (target, cell), E2L 4p^2+20p per (brick, cell), L2P 10p per
    target."""
    return (11.0 * stats["p2p_pairs"] + (16 * p + 8) * stats["e2p_pairs"]
            + (4 * p * p + 20 * p) * stats["e2l_pairs"] + 10.0 * p * stats["l2p_targets"])


def read_profile_traffic():
    """DRAM bytes per launch of k_force_eval from the committed ncu summary (or None)."""
    try:
        with open(PROFILE_TRAFFIC) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# ------------------------------------------------------------------------------- CPU reference
def cpu_reference_step(w, sample_blocks=128, threads=None):
    """One bounded step of the reference's CPU implementation (oracle/_ref: the reference's
    drivers compiled verbatim + the restated ISPC kernels, node capacity raised for large
    inputs): the full tree build plus the evaluation of `sample_blocks` evenly strided blocks,
    extrapolated linearly to all blocks.  Returns (seconds for the full workload, description).
    """
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # the checker / CPU baseline only
    nb = len(w["x0s"])
    stride = max(1, nb // sample_blocks)
    idx = np.arange(0, nb, stride)[:sample_blocks]
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    try:
        sys.stdout.flush()
        os.dup2(devnull, 1)   # the reference's force driver prints per-thread timers
        t0 = time.perf_counter()
        O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"][:0], w["y0s"][:0],
                     w["hs"][:0], mode="big")
        t1 = time.perf_counter()
        O.force_mrag(w["theta"], w["xs"], w["ys"], w["vs"], w["x0s"][idx], w["y0s"][idx],
                     w["hs"][idx], mode="big")
        t2 = time.perf_counter()
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    build = t1 - t0
    evals = max(t2 - t1 - build, 0.0)
    full = build + evals * nb / len(idx)
    desc = (f"full tree build ({len(w['xs'])} sources) + evaluation of {len(idx)} of {nb} "
            f"blocks (every {stride}th), evaluation time scaled by {nb}/{len(idx)}; "
            f"build {build:.2f} s, sampled evaluation {evals:.2f} s")
    return full, desc


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    w = make_workload(args.workload)
    if w["kind"] != "force":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference arm is implemented for the force_mrag workloads"}))
        return 0
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
        "data": "synthetic (seeded PCG64)",
        "config": {"workload": w["name"], "theta": w["theta"], "order": ORDER_FORCE,
                   "sources": len(w["xs"]), "targets": n_targets(w), "precision": "fp64",
                   "l2": "inputs larger than L2 (384 MB of sources)"},
        "cpu_baseline": {"value": val, "unit": "Mtargets/s", "cores": cores, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": val, "unit": "Mtargets/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------- GPU arm
def run_b200(args, ws, rank, local):
    import torch
    import treecodes as T

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA GPU")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = make_workload(args.workload, seed_offset=rank)
    kind = w["kind"]
    ctx = T.Context(device=local, precision=1 if args.precision == "mixed" else 0)
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
        print(json.dumps({"single": w["name"], "ms_per_step": (time.perf_counter() - t0) * 1e3
                          / max(args.steps, 1), "stats": ctx.stats()}))
        ctx.close()
        return 0

    # ---- device-resident throughput (value)
    for _ in range(max(args.warmup, 3)):
        solve()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    launches = 0
    for _ in range(args.steps):
        solve()
        launches += ctx.stats()["launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = sampler.stop()
    ms_local = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms_local, ws, dev)
    value = ws * m / (ms * 1e-3) / 1e6

    # ---- dominant kernel: evaluation launch timed with events on the library's stream
    ctx.set_timing(True)
    ev_ms = []
    for _ in range(3):
        solve()
        ev_ms.append(ctx.stats()["eval_ms"])
    st = ctx.stats()
    ctx.set_timing(False)
    eval_ms = statistics.median(ev_ms)
    flops = algorithmic_flops(st) if kind == "force" else None
    fp64_peak = T.measure_fma_peak(True)
    roofline = None
    if flops is not None:
        achieved = flops / (eval_ms * 1e-3) / 1e12
        roofline = {"kernel": "k_force_eval", "bound": "fp64", "achieved": achieved,
                    "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                    "traffic": read_profile_traffic(),
                    "peak_source": "measured FP64 FMA throughput of this GPU (tc_measure_fma_peak)",
                    "algorithmic_flops_per_launch": flops, "launch_ms": eval_ms,
                    "phase_ms": {k: st[k] for k in ("sort_ms", "tree_ms", "upward_ms",
                                                     "lists_ms", "eval_ms", "total_ms")}}

    # ---- accuracy vs the FP64 direct sum on a strided target subsample (GPU direct sum)
    acc = None
    if kind == "force":
        solve()
        torch.cuda.synchronize()
        step = max(1, m // args.accuracy_targets)
        idx = torch.arange(7, m, step, device=dev)[: args.accuracy_targets]
        ib, rem = idx // 1024, idx % 1024
        iy, ix = rem // 32, rem % 32
        xt = d["x0s"][ib] + ix.double() * d["hs"][ib]
        yt = d["y0s"][ib] + iy.double() * d["hs"][ib]
        rx = torch.empty(len(idx), dtype=torch.float64, device=dev)
        ry = torch.empty_like(rx)
        ctx.direct_force_device(d["xs"], d["ys"], d["vs"], xt, yt, rx, ry)
        gx, gy = out[0][idx], out[1][idx]
        num = torch.sqrt(((gx - rx) ** 2 + (gy - ry) ** 2).sum())
        den = torch.sqrt((rx ** 2 + ry ** 2).sum())
        acc = {"rel_l2_vs_fp64_direct": float(num / den),
               "max_abs_err": float(torch.maximum((gx - rx).abs(), (gy - ry).abs()).max()),
               "targets_sampled": int(len(idx))}

    # ---- end to end through the reference-compatible C entry point, pinned host buffers
    lib = T.load()
    import ctypes
    pin = {k: torch.as_tensor(w[k]).pin_memory() for k in ("xs", "ys", "vs", "x0s", "y0s", "hs")} \
        if kind == "force" else {k: torch.as_tensor(w[k]).pin_memory() for k in ("xs", "ys", "vs", "xt", "yt")}
    hout = [torch.empty(m, dtype=torch.float64).pin_memory() for _ in out]
    P = lambda t: ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))  # noqa: E731
    n = len(w["xs"])

    def solve_host():
        if kind == "force":
            lib.treecode_force_mrag(w["theta"], P(pin["xs"]), P(pin["ys"]), P(pin["vs"]), n,
                                    P(pin["x0s"]), P(pin["y0s"]), P(pin["hs"]), len(w["x0s"]),
                                    P(hout[0]), P(hout[1]))
        else:
            lib.treecode_potential(w["theta"], P(pin["xs"]), P(pin["ys"]), P(pin["vs"]), n,
                                   P(pin["xt"]), P(pin["yt"]), m, P(hout[0]))
        if lib.treecode_last_status() != 0:
            raise RuntimeError(lib.treecode_last_error().decode())

    for _ in range(max(args.warmup, 3)):
        solve_host()
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        solve_host()
    t1 = time.perf_counter()
    e2e_ms = max_over_ranks((t1 - t0) / args.steps * 1e3, ws, dev)
    h2d = sum(t.numel() * 8 for t in pin.values())
    d2h = sum(t.numel() * 8 for t in hout)
    e2e = {"value": ws * m / (e2e_ms * 1e-3) / 1e6, "unit": "Mtargets/s", "ms_per_step": e2e_ms,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "api": "treecode_force_mrag (C ABI, host pointers)" if kind == "force"
           else "treecode_potential (C ABI, host pointers)"}

    # ---- CPU baseline (rank 0, N = 1)
    cpu = None
    if rank == 0 and ws == 1 and kind == "force" and not args.no_cpu_baseline:
        try:
            t_full, desc = cpu_reference_step(w)
            cpu = {"value": m / t_full / 1e6, "unit": "Mtargets/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": desc}
        except Exception as exc:  # the oracle libraries are built in the source container
            cpu = {"value": None, "unit": "Mtargets/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": f"unavailable: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mtargets/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64; the reference's datasets are not available)",
            "config": {"workload": w["name"], "theta": w["theta"], "order": ORDER_FORCE
                       if kind == "force" else 12, "sources": len(w["xs"]), "targets": m,
                       "precision": "fp64", "parallelism": f"{ws} independent solves (one per GPU)",
                       "l2": "inputs larger than L2 (384 MB of sources per step)"},
            "accuracy": acc,
            "e2e": e2e,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches,
        }
        print(json.dumps(line))
    ctx.close()
    return 0


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
