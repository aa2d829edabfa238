"""Shared fixtures.  Tests marked `gpu` need a B200 and call the CUDA library
through its C ABI; everything else runs on the CPU (oracle, golden fixtures,
ABI exports, host-side argument checks, gloo multi-process logic)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def mxp():
    import openmxp_b200 as M
    M.lib()  # raises when libmxp.so is missing: no fallback
    return M


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    torch.cuda.init()
    return torch
