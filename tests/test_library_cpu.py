"""CPU-side checks of the product library and its host logic (no GPU compute):
the C-ABI shared object loads and exports every symbol the public header declares, the
Python binding covers the header, the library fails loudly without a GPU, the workload
generators and the MRAG output layout, and the benchmark's host-side arithmetic."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import treecodes as T
import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "treecodes_b200.h")


def header_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^TC_API\s+[\w\s\*]*?\b(\w+)\s*\(", text, re.M)))


def test_library_built_and_loads():
    assert os.path.exists(T.LIB_PATH), "build with make -C 2d-treecodes_b200"
    T.load()


def test_library_exports_every_header_symbol():
    names = header_symbols()
    assert "treecode_potential" in names and "treecode_force_mrag" in names
    lib = ctypes.CDLL(T.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", T.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    assert set(names) <= exported


def test_python_binding_covers_header():
    assert sorted(T.SIGNATURES) == header_symbols()


def test_supported_orders_list():
    """tc_supported_orders needs no device: the orders with kernel instances, the reference's
    defaults 12 and 24 among them."""
    orders = T.supported_orders()
    assert orders == sorted(orders) and {T.ORDER_POTENTIAL, T.ORDER_FORCE} <= set(orders)
    assert max(orders) <= 28   # E2L binomials C(2p-1, p-1) exact in FP64


def test_library_is_sm100a_build():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", T.LIB_PATH],
                         capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_fails_loudly_without_gpu():
    """No CPU fallback: with no visible GPU the reference entry point reports an error (status
    and stderr) instead of computing anything."""
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r);"
        "import treecodes as T\n"
        "x = np.random.random(64)\n"
        "try:\n"
        "    T.treecode_potential(0.5, x, x, x, x.copy(), x.copy())\n"
        "except T.TreecodeError as e:\n"
        "    print('STATUS', T.last_status()); sys.exit(0)\n"
        "sys.exit(3)\n" % os.path.join(ROOT, "2d-treecodes_b200"))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "STATUS 5" in r.stdout            # TC_ERR_NO_DEVICE
    assert "treecode_potential failed" in r.stderr


def test_workload_generators():
    w = W.uniform_potential(n=1000)
    assert len(w["xs"]) == 1000 and np.array_equal(w["xs"], w["xt"]) and w["xs"] is not w["xt"]
    assert w["xs"].min() >= 0 and w["xs"].max() < 1 and np.abs(w["vs"]).max() <= 1
    w = W.lamb_oseen_force(n=1000, blocks_per_side=4, h=1 / 128)
    assert len(w["x0s"]) == 16 and np.all(w["hs"] == 1 / 128)
    assert np.allclose(w["x0s"][:4], [0, 0.25, 0.5, 0.75]) and np.all(w["y0s"][:4] == 0)
    w = W.gaussian_mixture_potential(n=5000)
    assert w["xs"].min() >= 0 and w["xs"].max() < 1
    w = W.vortex_sheet_force(n=5000, blocks_per_side=4)
    assert np.all(w["vs"] > 0) and abs(w["ys"].mean() - 0.5) < 0.01
    # seeded: identical on every call
    assert np.array_equal(W.vortex_sheet_force(n=100, blocks_per_side=2)["ys"],
                          W.vortex_sheet_force(n=100, blocks_per_side=2)["ys"])


def test_mrag_output_layout():
    """Target (ix, iy) of block ib lives at ix + 32 * (iy + 32 * ib) (README.md:37)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    x0, y0, h = np.array([0.0, 10.0]), np.array([0.0, 20.0]), np.array([1.0, 0.5])
    xt, yt = O.mrag_targets(x0, y0, h)
    for ib, ix, iy in [(0, 3, 5), (1, 31, 0), (1, 2, 17)]:
        k = ix + 32 * (iy + 32 * ib)
        assert xt[k] == x0[ib] + ix * h[ib] and yt[k] == y0[ib] + iy * h[ib]


def test_bench_flop_model_and_profile_parse(tmp_path):
    sys.path.insert(0, ROOT)
    import bench
    st = dict(p2p_pairs=10, e2p_pairs=2, e2l_pairs=3, l2p_targets=64)
    p = 24
    fl = bench.algorithmic_flops(st)
    assert fl["k_force_near"] == 110
    assert fl["k_force_far"] == 2 * (16 * p + 8) + 3 * (4 * p * p + 20 * p) + 64 * 10 * p
    assert bench.algorithmic_flops(st, "potential") == {"k_potential_eval": 80 + 2 * (10 * 12 + 8)}
    (tmp_path / "k_force_far.vortex_sheet_force.txt").write_text(
        "kernel: k_force_far\ndram_bytes_per_launch: 123456 (read + write)\n")
    old = bench.PROFILES
    bench.PROFILES = str(tmp_path)
    try:
        assert bench.read_profile_traffic("k_force_far", False, "vortex_sheet_force") == 123456.0
        assert bench.read_profile_traffic("k_force_far", True, "vortex_sheet_force") is None
    finally:
        bench.PROFILES = old
    # the committed summaries of both kernels and both forms carry the traffic line
    for kernel in ("k_force_far", "k_force_near"):
        for mixed in (False, True):
            assert bench.read_profile_traffic(kernel, mixed, "vortex_sheet_force") > 0
