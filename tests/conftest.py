"""Shared test setup: import paths, the `gpu` marker, builds of the library and
the oracle."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "bvh-based-collision-detection-scheme_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (runs the CUDA path)")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def lib_built():
    import bvhcd
    if not os.path.exists(bvhcd.LIB_PATH):
        bvhcd.build()
    return bvhcd


@pytest.fixture(scope="session")
def cuda(lib_built):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")
    assert lib_built.device_check(0), "libbvhcd.so has no code for this device"
    return torch


@pytest.fixture(scope="session")
def cloth_c1():
    """128x128 cloth, 20 frames of the analytic fold (32,258 triangles)."""
    import scenes
    return scenes.cloth_fold_frames(128, 20)
