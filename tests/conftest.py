import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: full-size configurations (minutes)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "golden_vectors.json")) as f:
        return json.load(f)["cases"]


@pytest.fixture(scope="session")
def fmn():
    """The CUDA library; GPU tests fail loudly (no fallback) if it or the GPU is missing."""
    import fast_mul_ntt_b200 as m
    m.load_library()
    m.init(0)
    return m
