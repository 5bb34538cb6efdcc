"""The reference's test program on this library (run_dataset.py): generated files in the
reference's three formats are read, solved on the GPU through the reference-compatible entry
points, and checked against the GPU direct sum with main.cpp's rule; the printed error norms
agree with the oracle's (exact64 drivers, numpy direct sum of main.cpp:201-245)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [os.path.join(ROOT, "2d-treecodes_b200"), os.path.join(ROOT, "oracle"),
                os.path.join(ROOT, "tests")]

import datasets as D               # noqa: E402
import run_dataset as RD           # noqa: E402
from test_datasets import _write_reference_tree   # noqa: E402

pytestmark = pytest.mark.gpu


def test_reference_program_on_generated_files(tmp_path, monkeypatch):
    import oracle as O
    files = _write_reference_tree(tmp_path)
    monkeypatch.chdir(tmp_path)
    theta, tol = 0.5, 1e-7
    lines = []
    for path, kind in files:
        potential = kind == "potential"
        t = tol if potential else tol * 100
        res = RD.run_test(path, theta, t, potential=potential, mragfile=kind == "mrag",
                          out=lines.append)
        d = D.read(path, kind)
        idx = D.sample_indices(len(d["xt"]))
        if potential:
            want = [O.potential(theta, d["xs"], d["ys"], d["vs"], d["xt"], d["yt"])]
            refs = [D.direct_potential(d["xs"], d["ys"], d["vs"], d["xt"][idx], d["yt"][idx])]
        else:
            want = O.force_mrag(theta, d["xs"], d["ys"], d["vs"], d["x0s"], d["y0s"], d["hs"])
            refs = D.direct_force(d["xs"], d["ys"], d["vs"], d["xt"][idx], d["yt"][idx])
        assert len(res["checks"]) == len(want)
        for c, w, ref in zip(res["checks"], want, refs):
            assert c["ok"]
            o = D.check(ref, w[idx], t)
            # the GPU results equal the oracle's to ~1e-12 relative; the norms measure errors
            # a few orders larger, so they agree to a few digits
            scale = np.abs(ref).max()
            assert abs(c["linf_abs"] - o["linf_abs"]) <= 1e-2 * o["linf_abs"] + 1e-12 * scale
    assert sum("TEST PASSED." in l for l in lines) == 3


def test_failing_check_is_reported(tmp_path, monkeypatch):
    files = _write_reference_tree(tmp_path)
    monkeypatch.chdir(tmp_path)
    path, _ = files[1]
    # the force at theta 1 is accurate to ~1e-5, far from 100 x 1e-12: the program reports
    # the failure and exits with status 1
    assert RD.main(["1.0", "1e-12", "--file", f"{path}:V"]) == 1
