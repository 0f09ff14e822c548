"""Test configuration: import paths, the `gpu` marker and shared contexts."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "qsm.rs_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libqsmgpu.so")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx64():
    if not _cuda_available():
        pytest.fail("GPU test run without a CUDA device")
    import qsmgpu
    c = qsmgpu.Context(0, "f64")
    yield c
    c.close()


@pytest.fixture(scope="session")
def ctx32():
    if not _cuda_available():
        pytest.fail("GPU test run without a CUDA device")
    import qsmgpu
    c = qsmgpu.Context(0, "mixed")
    yield c
    c.close()
