import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); runs through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def renderer():
    import torch  # noqa: F401  (device presence check only)
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a visible CUDA device")
    from vork_b200 import Renderer
    from vork_b200.build import build
    build()
    r = Renderer(0)
    yield r
    r.close()


@pytest.fixture(scope="session")
def small_scene():
    from vork_b200 import scene
    return scene.spheres_scene()
