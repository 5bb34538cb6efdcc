"""CPU tests of the request server's scheduling (2d-treecodes_b200/csrc/server.cu).

server.cu talks to the solver only through the public context API, so it is linked here
against a stand-in for that API (tests/server_mock/mock_api.cpp) whose solves sleep, mark their
outputs and grow their context's memory figure.  Random streams then check admission under a
device-memory budget, eviction of resident clients, per-client ordering, completion of every
request and the absence of leaked contexts -- including streams whose contexts outgrow the
admission estimate, where the server must still make progress."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MOCK = os.path.join(ROOT, "tests", "server_mock")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc is needed to compile server.cu")
    out = tmp_path_factory.mktemp("server_mock") / "server_mock"
    cmd = [nvcc, "-O1", "--std=c++17", "-I" + os.path.join(ROOT, "include"),
           "-I" + os.path.join(ROOT, "2d-treecodes_b200", "csrc"),
           os.path.join(ROOT, "2d-treecodes_b200", "csrc", "server.cu"),
           os.path.join(MOCK, "mock_api.cpp"), os.path.join(MOCK, "mock_main.cpp"),
           "-o", str(out), "-lpthread"]
    subprocess.run(cmd, check=True, capture_output=True)
    return str(out)


@pytest.mark.parametrize("lo,hi,seed", [(0.9, 0.9, 1), (0.5, 1.0, 2), (0.5, 3.0, 3)])
def test_random_streams(harness, lo, hi, seed):
    r = subprocess.run([harness, "40", str(lo), str(hi), str(seed)], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
