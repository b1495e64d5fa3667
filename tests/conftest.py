"""Shared fixtures.  GPU tests carry ``@pytest.mark.gpu``; everything else runs
on the CPU.  The CPU checkers (oracle/pyoracle.py) are test infrastructure."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from pyoracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from pyoracle import Reference

    if not Reference.available():
        pytest.skip("reference native backend (oracle/_ref) not built")
    return Reference()


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from axhel_b200 import capi

    capi.lib()
    return capi
