"""Test configuration: import paths for the package and the oracle, and the `gpu` marker.

`-m "not gpu"` runs the oracle checks, host logic and library-loading tests on the CPU;
`-m gpu` runs the parity tests that call the CUDA library through its C ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "2d-treecodes_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200 / sm_100a)")


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch
    import treecodes
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    torch.cuda.init()
    ctx = treecodes.Context(device=0)
    yield ctx
    ctx.close()
