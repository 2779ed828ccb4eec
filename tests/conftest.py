"""Shared test setup: import paths, the ``gpu`` marker, the parity case list.

``-m "not gpu"`` runs on a CPU-only machine: the oracle (CPU restatement of the reference
algorithm) against known answers and committed golden fixtures, host-side logic, and the C-ABI
library's exports.  ``-m gpu`` runs the CUDA path through the C-ABI against the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "opencfd-ec_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); runs the product path")


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    oracle_py.build()
    return oracle_py


@pytest.fixture(scope="session")
def gpu():
    """The product library on a GPU.  Fails (never skips) when the library or the GPU is missing."""
    import torch
    from ocfd_b200 import build, capi
    if not os.path.exists(capi.LIB_PATH):
        build.build()
    assert torch.cuda.is_available(), "gpu tests need a CUDA device"
    torch.cuda.init()
    return capi
