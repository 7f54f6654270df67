import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    # build the native library and the oracle once per session (no GPU needed)
    import __graft_entry__

    __graft_entry__._load_build_module().build()
    import oracle

    oracle.build()
    oracle.build_reference()


@pytest.fixture(scope="session")
def menger_scene():
    import libsvo_b200 as L

    return L.Scene.menger(level=5, depth=8, seed=1)


@pytest.fixture(scope="session")
def small_menger_scene():
    import libsvo_b200 as L

    return L.Scene.menger(level=3, depth=5, seed=7)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
