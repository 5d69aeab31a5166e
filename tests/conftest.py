import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Build (or reuse) the engine library and the oracle once per session."""
    from axisem3d_b200.build import build
    import oracle
    build()
    oracle.build()
    return True


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
