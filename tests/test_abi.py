"""The C-ABI library loads and exports every symbol include/solargpu_b200.h
declares, plus the reference's own C++ entry points (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT, _has_gpu

HEADER = os.path.join(ROOT, "include", "solargpu_b200.h")
# Mangled names of include/solar_gpu_api.h:37-54 in the reference.
CXX_SYMBOLS = [
    "_ZN9solar_gpu27uncompressed_gpu_irradianceEPKfiiiiPKiS1_fRKSt6vectorISt5tupleIJffEESaIS6_EERKS4_IfSaIfEESE_S1_S1_Pf",
    "_ZN9solar_gpu25compressed_gpu_irradianceEPKfiiiiPKiS1_fRKSt6vectorISt5tupleIJffEESaIS6_EERKS4_IfSaIfEESE_S1_S1_Pf",
]


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(solar_gpu_\w+)\s*\(", text)))


def test_header_declares_drop_in_pair():
    names = declared_functions()
    assert "solar_gpu_uncompressed_gpu_irradiance" in names
    assert "solar_gpu_compressed_gpu_irradiance" in names


def test_library_exports_every_declared_symbol(cuda_lib):
    for name in declared_functions():
        assert hasattr(cuda_lib, name), name


def test_library_exports_reference_cxx_entry_points(cuda_lib):
    from solargpu_b200 import api
    out = subprocess.run(["nm", "-D", "--defined-only", api.LIB_PATH], capture_output=True, text=True).stdout
    for sym in CXX_SYMBOLS:
        assert sym in out


def test_default_options(cuda_lib):
    from solargpu_b200 import api
    o = api.options()
    assert (o.neighbor_format, o.hour_block, o.accumulation, o.reflection) == (0, 256, 0, 0)
    assert (o.group_size, o.use_graph, o.chunk_voxels) == (128, 1, 0)


def test_bad_options_are_rejected_before_device_work(cuda_lib):
    """Argument errors come back as return codes (the reference exits)."""
    from solargpu_b200 import api
    with pytest.raises(TypeError):
        api.options(no_such_option=1)


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_create_without_device_returns_error_code(cuda_lib):
    from solargpu_b200 import api
    h = C.c_void_p()
    rc = cuda_lib.solar_gpu_create(0, C.byref(h))
    assert rc == -3
    assert b"no CUDA device" in cuda_lib.solar_gpu_last_error()


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_drop_in_without_device_raises_not_falls_back(cuda_lib, scene64):
    from solargpu_b200 import api
    out = __import__("numpy").zeros(scene64.num_total, "float32")
    with pytest.raises(api.SolarGPUError):
        api.uncompressed_gpu_irradiance(scene64.grid, scene64.width, scene64.height, scene64.num_total,
                                        scene64.num_top, scene64.pixel_parent, scene64.wall_z,
                                        scene64.max_height, scene64.sun, scene64.direct, scene64.diffuse,
                                        scene64.slopes, scene64.aspects, out)


def test_short_hourly_series_rejected(cuda_lib, scene64):
    from solargpu_b200 import api
    import numpy as np
    out = np.zeros(scene64.num_total, np.float32)
    with pytest.raises(api.SolarGPUError) as e:
        api.uncompressed_gpu_irradiance(scene64.grid, scene64.width, scene64.height, scene64.num_total,
                                        scene64.num_top, scene64.pixel_parent, scene64.wall_z,
                                        scene64.max_height, scene64.sun[:100], scene64.direct, scene64.diffuse,
                                        scene64.slopes, scene64.aspects, out)
    assert e.value.code == -1
