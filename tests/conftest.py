import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "qumasun-workshop-template_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def qsb():
    """The product binding; its import fails loudly when the CUDA library is missing."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import qsb as mod
    return mod


@pytest.fixture(scope="session")
def qsb_host():
    """The product binding for host-only entry points (no device needed)."""
    import qsb as mod
    return mod
