"""Output writers of the annual irradiance path (caller side, host memory).

* ``write_voxel_dump`` writes the reference CLI's voxel dump
  (``src/main.cpp:44-67``, ``<dsm>_voxels.bin``): int32 num_total, int32
  num_top, then per voxel four float32 values, its cell's x and y, its height
  z (the cell height for a top voxel, its wall height for a wall voxel) and its
  annual irradiance (Wh/m^2), in voxel order.  ``read_voxel_dump`` reads it
  back.
* ``write_raster`` writes the top voxels' irradiance as a float32
  ``[height][width]`` array in raster order (``.npy``), the layout of the
  reference's GeoTIFF output (``src/main.cpp:176-178``); GeoTIFF itself needs
  libtiff, which this build does not use.
"""
from __future__ import annotations

import numpy as np

_HEADER = np.dtype([("num_total", "<i4"), ("num_top", "<i4")])
_RECORD = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("val", "<f4")])


def voxel_records(scene, irradiance: np.ndarray) -> np.ndarray:
    """The dump's per-voxel records (x, y, z, annual irradiance)."""
    N, T, W = scene.num_total, scene.num_top, scene.width
    irr = np.ascontiguousarray(irradiance, np.float32)
    if irr.shape != (N,):
        raise ValueError(f"irradiance has shape {irr.shape}, expected ({N},)")
    parent = np.asarray(scene.pixel_parent, np.int64)
    rec = np.empty(N, _RECORD)
    rec["x"] = (parent % W).astype(np.float32)
    rec["y"] = (parent // W).astype(np.float32)
    z = np.empty(N, np.float32)
    z[:T] = np.asarray(scene.grid, np.float32)[parent[:T]]
    z[T:] = np.asarray(scene.wall_z, np.float32)[: N - T]
    rec["z"] = z
    rec["val"] = irr
    return rec


def write_voxel_dump(path: str, scene, irradiance: np.ndarray) -> None:
    """Writes the reference's voxel dump format (src/main.cpp:44-67)."""
    hdr = np.array([(scene.num_total, scene.num_top)], _HEADER)
    rec = voxel_records(scene, irradiance)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(rec.tobytes())


def read_voxel_dump(path: str) -> tuple[int, int, np.ndarray]:
    """Returns (num_total, num_top, records with fields x, y, z, val)."""
    raw = np.fromfile(path, np.uint8)
    if raw.size < _HEADER.itemsize:
        raise ValueError("truncated voxel dump")
    hdr = raw[:_HEADER.itemsize].view(_HEADER)[0]
    n = int(hdr["num_total"])
    body = raw[_HEADER.itemsize:]
    if body.size != n * _RECORD.itemsize:
        raise ValueError(f"voxel dump holds {body.size} bytes of records, expected {n * _RECORD.itemsize}")
    return n, int(hdr["num_top"]), body.view(_RECORD)


def write_raster(path: str, scene, irradiance: np.ndarray) -> None:
    """Top voxels' annual irradiance as float32 [height][width] (.npy)."""
    irr = np.asarray(irradiance, np.float32)
    np.save(path, irr[: scene.num_top].reshape(scene.height, scene.width))


def write_geotiff(path: str, scene, irradiance: np.ndarray, meta=None) -> None:
    """Top voxels' annual irradiance as a single-band float32 GeoTIFF, with the
    input heightmap's georeferencing and compression when it came from one
    (src/main.cpp:178, src/geotiff_io.cpp:157-185), else pixel size 1 and
    no compression."""
    from solargpu_b200 import geotiff
    import dataclasses
    m = dataclasses.replace(meta) if meta is not None else geotiff.TiffMeta(pixel_scale=[1.0, 1.0, 0.0],
                                                                             tiepoints=[0.0] * 6)
    m.w, m.h = scene.width, scene.height
    if m.rows_per_strip <= 0 or m.rows_per_strip > m.h:
        m.rows_per_strip = m.h
    irr = np.asarray(irradiance, np.float32)
    geotiff.write_tiff(path, irr[: scene.num_top].reshape(scene.height, scene.width), m)
