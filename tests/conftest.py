"""Test configuration.

Markers: ``gpu`` for tests that need a CUDA device (the parity tests proper,
run on a B200); everything else runs on the CPU.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _gpu_count():
    try:
        import torch
        return torch.cuda.device_count() if torch.cuda.is_available() else 0
    except Exception:
        return 0


@pytest.fixture(scope="session")
def built_lib():
    """Builds libhm_erosion.so if needed and returns its path."""
    from highmap_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def gpu(built_lib):
    """A ready device; skips when the machine has no CUDA device."""
    if _gpu_count() == 0:
        pytest.skip("no CUDA device on this machine")
    from highmap_b200 import gpu as G
    assert G.init_opencl(), "hm_init failed on a machine with a CUDA device"
    return G
