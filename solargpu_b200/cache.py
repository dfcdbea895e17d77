"""On-disk cache of Stage 1 products (neighbor lists + shadow words).

Stage 1 (the DDA viewshed) depends only on the scene geometry (heights,
voxel layout, wall heights, max height) and on the sun positions (which fix
the sky bins and so the shadow-word layout); the hourly irradiance enters
only Stage 2/3.  A traced scene can therefore be saved once and re-run with
new hourly series through `Context.run_lists`, skipping the tracer:

    r = ctx.trace(scene, dev, neighbor_format=api.CSR)
    cache.save_lists("tile.npz", r, scene)
    ...
    lists = cache.load_lists("tile.npz", scene)        # checks the fingerprints
    ctx.run_lists(scene_with_new_tmy, dev, lists, out)

The file is a plain `.npz` (one list format, the shadow words, the sky-bin
counts and two SHA-256 fingerprints: geometry and sun positions).  The
reference has no counterpart: it traces on every run.
"""
from __future__ import annotations

import hashlib

import numpy as np

FORMAT_CSR, FORMAT_BARLE = 0, 1


def _sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode() + str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def scene_keys(scene) -> dict:
    """Fingerprints of what Stage 1 depends on."""
    geom = _sha(scene.grid, scene.pixel_parent, scene.wall_z,
                np.array([scene.width, scene.height, scene.num_total, scene.num_top], np.int64),
                np.array([scene.max_height], np.float32))
    return {"geometry": geom, "sun": _sha(np.asarray(scene.sun, np.float32)[:8760])}


def save_lists(path: str, lists: dict, scene, fmt: int | None = None) -> None:
    """Writes one list format of a `Context.trace()` result (CSR if present
    and `fmt` is None) with the shadow words and the scene fingerprints."""
    if fmt is None:
        fmt = FORMAT_CSR if "csr_off" in lists else FORMAT_BARLE
    if fmt == FORMAT_CSR:
        off, data = lists["csr_off"], lists["csr_ids"]
    else:
        off, data = lists["barle_off"], lists["barle"]
    keys = scene_keys(scene)
    np.savez(path, format=np.int32(fmt), offsets=np.asarray(off, np.int64),
             data=np.asarray(data, np.int32 if fmt == FORMAT_CSR else np.uint8),
             shadow=np.asarray(lists["shadow"], np.uint32),
             shadow_words=np.int32(lists["shadow_words"]), active_bins=np.int32(lists["active_bins"]),
             geometry_key=np.array(keys["geometry"]), sun_key=np.array(keys["sun"]))


def load_lists(path: str, scene=None) -> dict:
    """Reads a saved trace.  With `scene`, raises ValueError unless its
    geometry and sun positions are the ones the lists were traced with."""
    with np.load(path) as z:
        fmt = int(z["format"])
        if fmt not in (FORMAT_CSR, FORMAT_BARLE):
            raise ValueError(f"{path}: unknown list format {fmt}")
        off = z["offsets"]
        data = z["data"]
        if off.ndim != 1 or off.size < 1 or off[0] != 0 or off[-1] != data.size or np.any(np.diff(off) < 0):
            raise ValueError(f"{path}: offsets do not describe the data")
        out = {"shadow": z["shadow"], "shadow_words": int(z["shadow_words"]), "active_bins": int(z["active_bins"])}
        if out["shadow"].shape != (off.size - 1, out["shadow_words"]):
            raise ValueError(f"{path}: shadow words shape {out['shadow'].shape}")
        if fmt == FORMAT_CSR:
            out["csr_off"], out["csr_ids"] = off, data.astype(np.int32, copy=False)
        else:
            out["barle_off"], out["barle"] = off, data.astype(np.uint8, copy=False)
        if scene is not None:
            keys = scene_keys(scene)
            if str(z["geometry_key"]) != keys["geometry"]:
                raise ValueError(f"{path}: traced for a different geometry")
            if str(z["sun_key"]) != keys["sun"]:
                raise ValueError(f"{path}: traced for different sun positions")
    return out
