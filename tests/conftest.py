"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
import importlib
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "oracle") not in sys.path:
    sys.path.insert(0, str(ROOT / "oracle"))

PKG_NAME = "ads4-holographic-quantum-turbulence_b200"
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def hqt():
    """The package, with libhqt.so built if it is missing."""
    pkg = importlib.import_module(PKG_NAME)
    lib = ROOT / PKG_NAME / "libhqt.so"
    if not lib.exists():
        build = importlib.import_module(PKG_NAME + ".build")
        build.build()
    return pkg


@pytest.fixture(scope="session")
def oracle():
    import hqt_oracle
    return hqt_oracle


@pytest.fixture(scope="session")
def shipped_seed():
    import numpy as np
    d = np.load(GOLDEN / "seed_mu6_nz30_vy7.npz")
    return {k: d[k] for k in d.files}


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda(hqt):
    if not gpu_available():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    import torch
    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def dev(cuda, hqt):
    """(to_device, from_device) of the package's API."""
    api = importlib.import_module(hqt.__name__ + ".api")
    return api.to_device, api.from_device
