"""Shared test set-up: import paths, the gpu marker, scene fixtures."""
import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG = ROOT / "luminagi-cudaref_b200"
for p in (str(PKG), str(ROOT / "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _gpu_available() -> bool:
    """True when the CUDA driver reports at least one device (no torch import)."""
    import ctypes
    try:
        cuda = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return False
    if cuda.cuInit(0) != 0:
        return False
    n = ctypes.c_int(0)
    return cuda.cuDeviceGetCount(ctypes.byref(n)) == 0 and n.value > 0


HAVE_GPU = _gpu_available()


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def box_scene():
    import lumina
    return lumina.box_scene(1)


@pytest.fixture(scope="session")
def small_engine_scene():
    import lumina
    # Same construction as the 1.05M-triangle scene, scaled down (64x64 grids, 3-subdiv spheres).
    return lumina.engine_scene(seed=7, width=192, height=96, grid_n=64, sphere_subdiv=3)
