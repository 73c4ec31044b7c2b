"""Shared fixtures: seeded scenes, the oracle and the GPU library."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def tiny_scene():
    from tsr_b200 import scenes
    return scenes.sphere_scene(stride=16)


@pytest.fixture(scope="session")
def small_scene():
    from tsr_b200 import scenes
    return scenes.sphere_scene(stride=8)


@pytest.fixture(scope="session")
def csg_small():
    from tsr_b200 import scenes
    return scenes.csg_scene(n_target=30000, width=320, height=240, f=250.0, n_cams=24)
