"""Shared fixtures.  `-m "not gpu"` tests run on the CPU only (oracle, host
logic, library loading); `-m gpu` tests call the CUDA library through its
C ABI and compare with the oracle."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and calls the CUDA library")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def cuda_lib():
    """The product library, built in-tree if it is missing (never a fallback)."""
    from solargpu_b200 import api, build
    if not os.path.exists(api.LIB_PATH):
        build.build()
    return api.lib()


def load_scene(name: str):
    """Stored input arrays of a named scene (tests/golden/scene_<name>.npz)."""
    from solargpu_b200 import inputs
    path = os.path.join(GOLDEN, f"scene_{name}.npz")
    if os.path.exists(path):
        d = np.load(path)
        return inputs.scene_from_arrays(name, d, int(d["width"]), int(d["height"]))
    return inputs.make_scene(name)


@pytest.fixture(scope="session")
def scene64():
    return load_scene("dsm64")


@pytest.fixture(scope="session")
def scene160():
    return load_scene("dsm160")


_TRACE_CACHE: dict = {}


def oracle_trace(scene):
    """Oracle Stage 1 (CSR lists + shadow words), cached per scene."""
    from oracle import oracle as O
    if scene.name not in _TRACE_CACHE:
        bins = O.sky_bins(scene.sun)
        off, ids, sh = O.trace(scene, bins)
        _TRACE_CACHE[scene.name] = (bins, off, ids, sh)
    return _TRACE_CACHE[scene.name]


def device_arrays(scene):
    import torch
    dev = torch.device("cuda:0")
    return {
        "grid": torch.from_numpy(scene.grid).to(dev),
        "pixel_parent": torch.from_numpy(scene.pixel_parent).to(dev),
        "wall_z": torch.from_numpy(scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)).to(dev),
        "slopes": torch.from_numpy(scene.slopes).to(dev),
        "aspects": torch.from_numpy(scene.aspects).to(dev),
    }
