import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200; runs the CUDA path through the C ABI")


def _ensure_built():
    lib = os.path.join(ROOT, "vbd_tetmesh_b200", "libvbd_b200.so")
    orc = os.path.join(ROOT, "oracle", "libvbd_oracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "vbd_tetmesh_b200", "csrc")], check=True,
                       capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def gpu_device():
    """The CUDA device index for GPU tests (fails, never skips, when no B200 is present)."""
    import torch

    assert torch.cuda.is_available(), "GPU test collected on a machine without CUDA"
    major, minor = torch.cuda.get_device_capability(0)
    assert (major, minor) == (10, 0), f"expected a B200 (sm_100), got sm_{major}{minor}"
    return 0
