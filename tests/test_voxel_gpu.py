"""GPU voxelization (solar_gpu_voxelize) against the reference's own
voxelization (src/voxelization.cpp:10-97, run on the host and stored in
tests/golden/voxel_<name>.npz) and against the packed arrays the
caller-side restatement builds (solargpu_b200/inputs.py).

Wall counts, parents and heights are integer / exact float work: equal.
Angles come from CUDA's atan2f against the host library's: within 2e-6 rad."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_scene

pytestmark = pytest.mark.gpu
ANGLE_TOL = 2e-6


def _voxelize(scene):
    import torch
    from solargpu_b200 import api
    g = torch.from_numpy(scene.grid).cuda()
    with api.Context(0) as ctx:
        r = ctx.voxelize(g, scene.width, scene.height, 1.0)
    torch.cuda.synchronize()
    n, t = r["num_total"], r["num_top"]
    return (n, t, r["pixel_parent"].cpu().numpy(), r["wall_z"].cpu().numpy()[:n - t], r["slopes"].cpu().numpy(),
            r["aspects"].cpu().numpy())


@pytest.mark.parametrize("name", ["dsm64", "dsm160"])
def test_voxelize_matches_reference_voxelization(cuda_lib, name):
    s = load_scene(name)
    g = np.load(os.path.join(GOLDEN, f"voxel_{name}.npz"))
    n, t, par, wz, sl, asp = _voxelize(s)
    assert t == s.width * s.height and n - t == g["parent"].size
    np.testing.assert_array_equal(par[:t], np.arange(t))
    np.testing.assert_array_equal(par[t:], g["parent"])
    np.testing.assert_array_equal(wz, g["z"])
    assert np.abs(asp[t:] - g["aspect"]).max() <= ANGLE_TOL
    assert np.abs(sl[:t] - g["slope"]).max() <= ANGLE_TOL
    assert np.abs(asp[:t] - g["top_aspect"]).max() <= ANGLE_TOL
    assert np.all(sl[t:] == np.float32(np.pi) * np.float32(0.5))


def test_voxelize_city_matches_host_arrays(cuda_lib):
    """The 1024 x 1024 city (1.5 M voxels): the same packed arrays as the
    host restatement the benchmark feeds the entry points."""
    from solargpu_b200 import inputs
    s = inputs.make_scene("dsm1024")
    n, t, par, wz, sl, asp = _voxelize(s)
    assert (n, t) == (s.num_total, s.num_top)
    np.testing.assert_array_equal(par, s.pixel_parent)
    np.testing.assert_array_equal(wz, s.wall_z)
    assert np.abs(sl - s.slopes).max() <= ANGLE_TOL
    d = np.abs(asp - s.aspects)
    d = np.minimum(d, np.float32(2 * np.pi) - d)   # 0 and 2 pi are the same direction
    assert d.max() <= ANGLE_TOL
