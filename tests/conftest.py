"""Shared pytest setup.

Markers: `gpu` tests need a B200 and the built libphix_b200.so; everything
else runs on the CPU (oracle, golden vectors, host logic, symbol checks).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libphix_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference library compiled from its sources (oracle/_ref), if built."""
    from oracle.oracle import LIB_REF, Reference
    if not os.path.exists(LIB_REF):
        pytest.skip("oracle/_ref/libphix_ref.so not built (needs the reference tree)")
    return Reference()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test collected on a machine without CUDA")
    import phix_b200
    phix_b200.lib()
    return torch.device("cuda:0")


def rng(seed):
    return np.random.default_rng(seed)
