"""The reference's test program (main.cpp) run on this library.

Reads the reference's binary dataset files (``datasets.py``), solves them with the
reference-compatible entry points ``treecode_potential`` / ``treecode_force_mrag`` on the GPU,
and checks every 433rd target from the 8th on against an FP64 direct sum computed on the GPU
(``tc_direct_*_device``), with main.cpp's pass rule and printout (main.cpp:31-59, 62-270).

    python run_dataset.py [theta [tol [profile]]] [--file PATH:KIND ...]

``theta`` defaults to 1 and ``tol`` to 1e-8 as in main.cpp:275-286; the force tests use
100 x tol (main.cpp:314).  ``profile`` skips the check.  KIND is P (potential file), V
(velocity file), PV (both readings of one file) or M (MRAG file).  Without ``--file`` the
reference's own file list (main.cpp:325-343) is tried relative to the working directory,
and missing files are skipped with a warning, as main.cpp does.  Exit status 1 if a check
fails.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import datasets as D      # noqa: E402
import treecodes as T     # noqa: E402

# main.cpp:325-343: (path, MRAG file, tests)
REFERENCE_FILES = [
    ("testDiego/diegoBinaryN400", False, "P"),
    ("testDiego/diegoBinaryN2000", False, "P"),
    ("testDiego/diegoBinaryN12000", False, "P"),
    ("diegoVel/velocityPoissonFishLmax6", False, "V"),
    ("diegoVel/velocityPoissonCylUnif2048", False, "V"),
    ("diegoVel/velocityPoissonFishLmax8Early", False, "V"),
    ("diegoVel/velocityPoissonFishLmax8Late", False, "V"),
    ("testSid/diegoSolverCylUniform", True, "V"),
    ("testSid/diegoSolverAdaptiveGrid", True, "V"),
    ("testSid/diegoVelTestsDec10", True, "V"),
    ("testSid/diegoVelTestsDec14", True, "V"),
]


class CheckFailed(RuntimeError):
    pass


def _direct(kind, d, idx):
    """FP64 direct sums at the targets ``idx`` on the GPU."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    t = {k: torch.as_tensor(np.ascontiguousarray(d[k]), device=dev) for k in ("xs", "ys", "vs")}
    xt = torch.as_tensor(np.ascontiguousarray(d["xt"][idx]), device=dev)
    yt = torch.as_tensor(np.ascontiguousarray(d["yt"][idx]), device=dev)
    ctx = T.Context()
    try:
        if kind == "potential":
            out = torch.empty(len(idx), dtype=torch.float64, device=dev)
            ctx.direct_potential_device(t["xs"], t["ys"], t["vs"], xt, yt, out)
            torch.cuda.synchronize()
            return out.cpu().numpy(), None
        u = torch.empty(len(idx), dtype=torch.float64, device=dev)
        w = torch.empty_like(u)
        ctx.direct_force_device(t["xs"], t["ys"], t["vs"], xt, yt, u, w)
        torch.cuda.synchronize()
        return u.cpu().numpy(), w.cpu().numpy()
    finally:
        ctx.close()


def _report(r, ref, res, tol, out):
    for i in r["failures"]:
        err = ref[i] - res[i]
        rel = err / max(1e-6, max(abs(res[i]), abs(ref[i])))
        out(f"{i}: {res[i]:e} ref: {ref[i]:e} -> {err:e} {rel:e}")
    out(f"l-infinity errors: {r['linf_abs']:.3e} (absolute) {r['linf_rel']:.3e} (relative)")
    out(f"       l-1 errors: {r['l1_abs']:.3e} (absolute) {r['l1_rel']:.3e} (relative)")


def run_test(path, theta, tol, potential=True, verify=True, mragfile=False, out=print):
    """main.cpp's test() on one file; returns a dict of what it measured, raises CheckFailed."""
    kind = "potential" if potential else ("mrag" if mragfile else "velocity")
    d = D.read(path, kind)
    n, m = len(d["xs"]), len(d["xt"])
    if kind == "mrag":
        out(f"mrag file! {len(d['x0s'])} blocks")
    elif kind == "velocity":
        out(f"ndst: {m} i have found {len(d['x0s'])} blocks")
    out(f"Testing {'POTENTIAL' if potential else 'FORCE'} with {n} sources and {m} targets "
        f"(theta {theta:.3e})...")
    t0 = time.perf_counter()
    if potential:
        res = (T.treecode_potential(theta, d["xs"], d["ys"], d["vs"], d["xt"], d["yt"]),)
    else:
        res = T.treecode_force_mrag(theta, d["xs"], d["ys"], d["vs"], d["x0s"], d["y0s"], d["hs"])
    ms = (time.perf_counter() - t0) * 1e3
    out(f"solved in {ms:.2f} ms")
    result = {"nsources": n, "ntargets": m, "theta": theta, "ms": ms, "checks": []}
    if verify:
        idx = D.sample_indices(m)
        refs = _direct("potential" if potential else "force", d, idx)
        for ref, r in zip(refs, res):
            if ref is None:
                continue
            got = r[idx]
            c = D.check(ref, got, tol)
            _report(c, ref, got, tol, out)
            result["checks"].append(c)
            if not c["ok"]:
                raise CheckFailed(f"{path}: {len(c['failures'])} of {len(idx)} checked targets "
                                  f"exceed tol {tol:g}")
    out("TEST PASSED.")
    return result


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("theta", nargs="?", type=float, default=1.0)
    p.add_argument("tol", nargs="?", type=float, default=1e-8)
    p.add_argument("mode", nargs="?", default="", help="'profile' skips the check")
    p.add_argument("--file", action="append", default=[],
                   help="PATH:KIND with KIND in P, V, PV, M (repeatable)")
    a = p.parse_args(argv)
    verify = a.mode != "profile"
    files = []
    for spec in a.file:
        path, _, k = spec.rpartition(":")
        if not path or k not in ("P", "V", "PV", "M"):
            p.error(f"--file wants PATH:KIND with KIND in P, V, PV, M, not {spec!r}")
        files.append((path, k == "M", "V" if k == "M" else k))
    if not files:
        files = REFERENCE_FILES
    failed = 0
    for path, mragfile, tests in files:
        if not os.access(path, os.R_OK):
            print(f"WARNING: reference file <{path}> not found, i skip this test.")
            continue
        print(f"reading from <{path}> ...")
        try:
            if not mragfile and "P" in tests:
                run_test(path, a.theta, a.tol, True, verify)
            if "V" in tests:
                run_test(path, a.theta, a.tol * 100, False, verify, mragfile)
        except (CheckFailed, D.DatasetError) as e:
            print(f"FAILED: {e}")
            failed += 1
    return 1 if failed else 0


if __name__ == "__main__":
    sys.exit(main())
