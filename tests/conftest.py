import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REFERENCE = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libdcxgpu.so")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    from distributed_suffix_sorting_evaluation_b200 import Context
    if not gpu_available():
        pytest.skip("no GPU")
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    return O


def reference_file(*parts):
    """Path of a file in the reference tree, or skip when the tree is absent."""
    p = os.path.join(REFERENCE, *parts)
    if not os.path.exists(p):
        pytest.skip("reference tree not mounted")
    return p


def random_text(n, sigma, seed, offset=65):
    rng = np.random.default_rng(seed)
    return rng.integers(offset, offset + sigma, n).astype(np.uint8)
