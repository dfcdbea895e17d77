"""GeoTIFF heightmaps and rasters (solargpu_b200/geotiff.py), the files the
reference CLI reads and writes with libtiff (src/geotiff_io.cpp:50-185).

The codec is checked three ways: its own round trip over every layout it
writes (strips, tiles, each compression and predictor); PIL, whose TIFF
decoder is libtiff, reading the files it writes and it reading PIL's; and the
reference's own test heightmap (tiled, Deflate, floating-point predictor, as
GDAL writes them) against the digest of PIL's decoding in
tests/golden/ref_dsm_tiff.json."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

REF = os.environ.get("SOLARGPU_REFERENCE", "/root/reference")
REF_DSM = os.path.join(REF, "test_data", "dsm_heightmap.tiff")


def _meta(g, w, h, comp, rps=0):
    return g.TiffMeta(w=w, h=h, compression=comp, rows_per_strip=rps, pixel_scale=[0.5, 0.5, 0.0],
                      tiepoints=[0.0, 0.0, 0.0, 545000.5, 156000.25, 0.0], geo_keys=[1, 1, 0, 1, 1024, 0, 1, 1],
                      geo_doubles=[6378137.0], geo_ascii="MGI / Slovenia Grid|")


@pytest.mark.parametrize("comp", [1, 5, 8, 32946])
@pytest.mark.parametrize("pred", [1, 2, 3])
@pytest.mark.parametrize("tile,rps", [(0, 0), (0, 7), (16, 0)])
def test_round_trip_every_layout(tmp_path, comp, pred, tile, rps):
    from solargpu_b200 import geotiff as g
    rng = np.random.default_rng(comp * 10 + pred)
    a = (rng.standard_normal((37, 53)) * 100).astype(np.float32)
    a[3, 4], a[5, 6] = np.float32(-9999.0), np.float32(np.inf)
    m = _meta(g, 53, 37, comp, rps)
    p = str(tmp_path / "r.tif")
    g.write_tiff(p, a, m, tile=tile, predictor=pred)
    b, m2 = g.read_tiff(p)
    assert np.array_equal(a.view(np.int32), b.view(np.int32))
    for k in ("w", "h", "compression", "pixel_scale", "tiepoints", "geo_keys", "geo_doubles", "geo_ascii"):
        assert getattr(m2, k) == getattr(m, k), k
    pil = pytest.importorskip("PIL.Image")
    if comp != 1 or pred == 1:   # libtiff applies a predictor only to compressed data
        c = np.array(pil.open(p), dtype=np.float32)
        assert np.array_equal(a.view(np.int32), c.view(np.int32))


@pytest.mark.parametrize("compression", ["raw", "tiff_lzw", "tiff_adobe_deflate"])
def test_reads_files_written_by_libtiff(tmp_path, compression):
    pil = pytest.importorskip("PIL.Image")
    from solargpu_b200 import geotiff as g
    a = (np.random.default_rng(5).standard_normal((61, 47)) * 30 + 300).astype(np.float32)
    p = str(tmp_path / "pil.tif")
    pil.fromarray(a, mode="F").save(p, compression=compression)
    b, m = g.read_tiff(p)
    assert (m.w, m.h) == (47, 61)
    assert np.array_equal(a.view(np.int32), b.view(np.int32))


def test_lzw_codec_round_trip():
    from solargpu_b200 import geotiff as g
    rng = np.random.default_rng(1)
    for data in (b"", b"a", bytes(70000), rng.integers(0, 256, 200000, dtype=np.uint8).tobytes(),
                 bytes(rng.integers(0, 4, 300000, dtype=np.uint8))):
        assert g.lzw_decode(g.lzw_encode(data)) == data


def test_rejects_non_float_rasters(tmp_path):
    pil = pytest.importorskip("PIL.Image")
    from solargpu_b200 import geotiff as g
    p = str(tmp_path / "u8.tif")
    pil.fromarray(np.zeros((4, 4), np.uint8)).save(p)
    with pytest.raises(g.TiffError, match="Expected 32-bit float TIFF"):
        g.read_tiff(p)


@pytest.mark.skipif(not os.path.exists(REF_DSM), reason="reference test heightmap not present")
def test_reads_reference_heightmap():
    """test_data/dsm_heightmap.tiff of the reference: 366 x 320, tiles of
    256, Deflate, floating-point predictor, GDAL no-data tag."""
    from solargpu_b200 import geotiff as g
    with open(os.path.join(GOLDEN, "ref_dsm_tiff.json")) as f:
        want = json.load(f)
    a, m = g.read_tiff(REF_DSM)
    assert list(a.shape) == want["shape"]
    assert hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest() == want["sha256_float32"]
    assert m.pixel_scale == want["pixel_scale"] and m.tiepoints == want["tiepoints"]
    assert m.nodata == want["nodata"] and m.compression == want["compression"]


def test_raster_writer_carries_georeferencing(tmp_path):
    """The CLI's output raster: top voxels in raster order, the input's
    georeferencing and compression, one strip (as the reference writes it)."""
    from solargpu_b200 import geotiff as g
    from solargpu_b200 import inputs, outputs
    rng = np.random.default_rng(2)
    h = (rng.random((24, 20)) * 5).astype(np.float32)
    h[8:14, 6:12] += 12.0
    m = _meta(g, 20, 24, 8)
    s = inputs.scene_from_heightmap("t", h, 0.5, 15.592, 46.543, 1)
    irr = rng.random(s.num_total).astype(np.float32) * 1e6
    p = str(tmp_path / "out.tiff")
    outputs.write_geotiff(p, s, irr, m)
    b, m2 = g.read_tiff(p)
    assert np.array_equal(b.ravel(), irr[:s.num_top])
    assert (m2.pixel_scale, m2.tiepoints, m2.geo_ascii, m2.compression, m2.rows_per_strip) == \
        (m.pixel_scale, m.tiepoints, m.geo_ascii, 8, 24)


def test_scene_from_heightmap_uses_pixel_size():
    """Walls and top slopes use the raster's pixel size (src/main.cpp:104-106)."""
    from solargpu_b200 import inputs
    h = np.zeros((16, 16), np.float32)
    h[5:10, 5:10] = 6.0
    s1 = inputs.scene_from_heightmap("a", h, 1.0, 15.0, 46.0, 1)
    s2 = inputs.scene_from_heightmap("b", h, 2.0, 15.0, 46.0, 1)
    n1 = s1.num_total - s1.num_top
    n2 = s2.num_total - s2.num_top
    assert n1 > 0 and n2 > 0 and n2 < n1                  # 2 m voxels: fewer wall voxels per drop
    assert not np.array_equal(s1.slopes[:s1.num_top], s2.slopes[:s2.num_top])


@pytest.mark.gpu
def test_cli_on_geotiff_heightmap(cuda_lib, tmp_path):
    """The CLI end to end on a GeoTIFF heightmap written as GDAL writes them
    (tiles, Deflate, floating-point predictor): its output GeoTIFF holds the
    same irradiance as the library run on the same inputs, with the input's
    georeferencing."""
    import subprocess
    import sys
    import torch
    from conftest import ROOT, device_arrays, load_scene
    from solargpu_b200 import api, geotiff as g, inputs
    h = load_scene("dsm64").grid.reshape(64, 64) + np.float32(300.0)   # absolute elevations, as a DSM
    m = _meta(g, 64, 64, 8)
    m.pixel_scale = [1.0, 1.0, 0.0]
    src, dst = str(tmp_path / "dsm.tif"), str(tmp_path / "out.tiff")
    g.write_tiff(src, h, m, tile=32, predictor=3)
    p = subprocess.run([sys.executable, "-m", "solargpu_b200.run", "--dsm", src, "--lon", "15.592", "--lat",
                        "46.543", "--tz", "1", "--runs", "1", "--out", dst], cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    got, m2 = g.read_tiff(dst)
    s = inputs.scene_from_heightmap("dsm.tif", h, 1.0, 15.592, 46.543, 1)
    out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
    with api.Context(0) as c:
        c.run_device(s, device_arrays(s), out, neighbor_format=0, hour_block=256, group_size=128, accumulation=1,
                     use_graph=0, time_kernels=1)
    want = out.cpu().numpy()[:s.num_top].reshape(64, 64)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
    assert (m2.tiepoints, m2.geo_keys, m2.geo_ascii) == (m.tiepoints, m.geo_keys, m.geo_ascii)
