import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) and the built CUDA library")
    config.addinivalue_line("markers", "slow: longer oracle runs")


def pytest_collection_modifyitems(config, items):
    # GPU tests fail loudly (no skip) when selected with -m gpu on a machine
    # without a GPU; when not selected they are simply deselected.
    pass


@pytest.fixture(scope="session")
def gpu_lib():
    import forestclaw_b200 as fcb
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return fcb.lib()
