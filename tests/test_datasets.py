"""The reference's dataset files (main.cpp:62-172): byte layout, the three readings, the check
rule, and a pin against the reference's own test program (main.cpp compiled against the
oracle drivers, oracle/_ref/ref_main) on generated files."""
import math
import os
import re
import struct
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [os.path.join(ROOT, "2d-treecodes_b200"), os.path.join(ROOT, "oracle")]

import datasets as D          # noqa: E402
import run_dataset as RD      # noqa: E402

REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "ref_main")


def _sources(n, seed):
    r = np.random.default_rng(seed)
    return r.random(n), r.random(n), r.uniform(-1, 1, n) / n


def _blocks(g):
    x0, y0 = np.meshgrid(np.arange(g) / g, np.arange(g) / g)
    return x0.ravel(), y0.ravel(), np.full(g * g, 1.0 / (32 * g))


def test_potential_file_bytes_and_round_trip(tmp_path):
    xs, ys, vs = np.array([0.1, 0.2]), np.array([0.3, 0.4]), np.array([1.0, -2.0])
    xt, yt, ref = np.array([0.5]), np.array([0.6]), np.array([7.0])
    p = tmp_path / "pot"
    D.write_potential(p, xs, ys, vs, xt, yt, ref)
    want = (struct.pack("<i", 2) + struct.pack("<6d", 0.1, 0.2, 0.3, 0.4, 1.0, -2.0) +
            struct.pack("<i", 1) + struct.pack("<3d", 0.5, 0.6, 7.0))
    assert p.read_bytes() == want
    d = D.read(p, "potential")
    for k, a in (("xs", xs), ("ys", ys), ("vs", vs), ("xt", xt), ("yt", yt), ("ref", ref)):
        assert np.array_equal(d[k], a)


def test_velocity_reading_transforms_reference_and_derives_blocks(tmp_path):
    x0, y0, hs = _blocks(2)
    xt, yt = D.block_targets(x0, y0, hs)
    xs, ys, vs = _sources(50, 1)
    ref, ref1 = np.arange(len(xt), dtype=float), -np.arange(len(xt), dtype=float) / 3
    p = tmp_path / "vel"
    D.write_potential(p, xs, ys, vs, xt, yt, ref, ref1)
    d = D.read(p, "velocity")
    # main.cpp:130-141: (x, y) reference = (-2 pi ref1, 2 pi ref)
    assert np.array_equal(d["uref"], -(ref1 * (2 * math.pi)))
    assert np.array_equal(d["vref"], ref * (2 * math.pi))
    # main.cpp:166-171: origins from the first point of each block, spacing from the second
    assert np.array_equal(d["x0s"], x0) and np.array_equal(d["y0s"], y0)
    assert np.allclose(d["hs"], hs, rtol=0, atol=1e-15)
    # the same file still reads as a potential file (main.cpp's PV tests)
    assert np.array_equal(D.read(p, "potential")["ref"], ref)


def test_mrag_file_target_layout(tmp_path):
    x0, y0, hs = np.array([0.0, 1.0]), np.array([2.0, 3.0]), np.array([0.5, 0.25])
    xs, ys, vs = _sources(10, 2)
    p = tmp_path / "mrag"
    D.write_mrag(p, xs, ys, vs, x0, y0, hs)
    d = D.read(p, "mrag")
    assert np.array_equal(d["x0s"], x0) and np.array_equal(d["hs"], hs)
    # target (ix, iy) of block b at ix + 32 (iy + 32 b), = (x0 + ix h, y0 + iy h)
    for b, ix, iy in ((0, 0, 0), (0, 31, 0), (0, 3, 17), (1, 5, 31)):
        k = ix + 32 * (iy + 32 * b)
        assert d["xt"][k] == x0[b] + ix * hs[b] and d["yt"][k] == y0[b] + iy * hs[b]


def test_malformed_files_are_rejected(tmp_path):
    p = tmp_path / "short"
    p.write_bytes(struct.pack("<i", 4) + struct.pack("<3d", 1, 2, 3))
    with pytest.raises(D.DatasetError):
        D.read(p, "potential")
    q = tmp_path / "notblocks"
    xs, ys, vs = _sources(5, 3)
    D.write_potential(q, xs, ys, vs, np.zeros(100), np.zeros(100), np.zeros(100), np.zeros(100))
    with pytest.raises(D.DatasetError, match="blocks"):
        D.read(q, "velocity")
    r = tmp_path / "neg"
    r.write_bytes(struct.pack("<i", -1))
    with pytest.raises(D.DatasetError, match="negative"):
        D.read(r, "potential")


def test_check_rule_and_samples():
    # pass if relative OR absolute error is below tol (main.cpp:44-48)
    ref = np.array([1.0, 1e-9, 100.0, 0.0])
    ok = D.check(ref, ref * (1 + 5e-9), 1e-8)
    assert ok["ok"]
    bad = D.check(ref, np.array([1.0 + 2e-8, 1e-9, 100.0 + 2e-6, 0.0]), 1e-8)
    assert bad["failures"] == [0, 2]
    # tiny values: relative error is taken against max(1e-6, |value|), so 5e-9 absolute passes
    assert D.check(np.array([1e-9]), np.array([6e-9]), 1e-8)["ok"]
    assert D.sample_indices(1000).tolist() == [7, 440, 873]


def test_missing_reference_files_are_skipped(tmp_path, capsys, monkeypatch):
    monkeypatch.chdir(tmp_path)
    assert RD.main([]) == 0
    out = capsys.readouterr().out
    assert out.count("WARNING: reference file") == len(RD.REFERENCE_FILES)


def _write_reference_tree(root):
    """Generated files under the reference program's own names (main.cpp:325-343)."""
    (root / "testDiego").mkdir()
    (root / "diegoVel").mkdir()
    (root / "testSid").mkdir()
    xs, ys, vs = _sources(400, 11)
    r = np.random.default_rng(12)
    xt, yt = r.random(3000), r.random(3000)
    D.write_potential(root / "testDiego" / "diegoBinaryN400", xs, ys, vs, xt, yt, np.zeros(3000))
    x0, y0, hs = _blocks(2)
    xs, ys, vs = _sources(12000, 13)
    xt, yt = D.block_targets(x0, y0, hs)
    D.write_potential(root / "diegoVel" / "velocityPoissonFishLmax6", xs, ys, vs, xt, yt,
                      np.zeros(len(xt)), np.zeros(len(xt)))
    xs, ys, vs = _sources(9000, 14)
    D.write_mrag(root / "testSid" / "diegoSolverCylUniform", xs, ys, vs, x0, y0, hs)
    return [("testDiego/diegoBinaryN400", "potential"),
            ("diegoVel/velocityPoissonFishLmax6", "velocity"),
            ("testSid/diegoSolverCylUniform", "mrag")]


def _parse(out):
    """(nsources, ntargets, theta, linf_abs, linf_rel, l1_abs, l1_rel) of each check printed."""
    tests = []
    for m in re.finditer(r"Testing (\w+) with (\d+) sources and (\d+) targets \(theta ([\d.e+-]+)\)",
                         out):
        tests.append({"kind": m.group(1), "n": int(m.group(2)), "m": int(m.group(3)),
                      "theta": float(m.group(4)), "pos": m.end(), "norms": []})
    norms = [(m.start(), tuple(map(float, m.groups()))) for m in re.finditer(
        r"l-infinity errors: ([\d.e+-]+) \(absolute\) ([\d.e+-]+) \(relative\)\n\s+l-1 errors: "
        r"([\d.e+-]+) \(absolute\) ([\d.e+-]+) \(relative\)", out)]
    for i, t in enumerate(tests):
        end = tests[i + 1]["pos"] if i + 1 < len(tests) else len(out)
        t["norms"] = [v for p, v in norms if t["pos"] <= p < end]
    return tests


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="oracle/_ref/ref_main not built")
def test_reader_and_check_match_the_reference_program(tmp_path):
    """The reference's main.cpp, run on generated files, reads the same sizes and prints the same
    error norms as this module's reader + check rule applied to the same drivers (the oracle's
    faithful build, which ref_main links) and the direct sum of main.cpp:201-245."""
    import oracle as O
    files = _write_reference_tree(tmp_path)
    theta, tol = 0.5, 1e-5
    run = subprocess.run([REF_MAIN, str(theta), str(tol)], cwd=tmp_path, capture_output=True,
                         text=True, timeout=600)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr[-2000:]
    assert run.stdout.count("TEST PASSED.") == 3
    ref_tests = _parse(run.stdout)
    assert [t["kind"] for t in ref_tests] == ["POTENTIAL", "FORCE", "FORCE"]
    for (path, kind), rt in zip(files, ref_tests):
        d = D.read(tmp_path / path, kind)
        assert (rt["n"], rt["m"], rt["theta"]) == (len(d["xs"]), len(d["xt"]), theta)
        idx = D.sample_indices(len(d["xt"]))
        if kind == "potential":
            res = [O.potential(theta, d["xs"], d["ys"], d["vs"], d["xt"], d["yt"], mode="faithful")]
            refs = [D.direct_potential(d["xs"], d["ys"], d["vs"], d["xt"][idx], d["yt"][idx])]
            t = tol
        else:
            res = O.force_mrag(theta, d["xs"], d["ys"], d["vs"], d["x0s"], d["y0s"], d["hs"],
                               mode="faithful")
            refs = D.direct_force(d["xs"], d["ys"], d["vs"], d["xt"][idx], d["yt"][idx])
            t = tol * 100
        assert len(rt["norms"]) == len(res)
        for r, ref, printed in zip(res, refs, rt["norms"]):
            c = D.check(ref, r[idx], t)
            assert c["ok"]
            mine = (c["linf_abs"], c["linf_rel"], c["l1_abs"], c["l1_rel"])
            # printed with 4 significant digits; the direct sums differ only in summation order
            assert np.allclose(mine, printed, rtol=3e-3, atol=0), (path, mine, printed)
