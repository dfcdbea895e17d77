"""Generates the golden fixtures under tests/golden/ from the reference's own
code, compiled from its sources by oracle/Makefile:

  host   (this container, needs the reference tree for oracle/_ref/libref_host.so)
    scene_<name>.npz      stored input arrays of the small scenes
    barle_golden.npz      id lists and the reference encoder's bytes
                          (src/barle_compression.cpp:156-187)
    sky_<name>.npz        reference sky bins (src/sky_bins.cpp:9-52)
    voxel_<name>.npz      reference voxelization (src/voxelization.cpp:10-97)
  gpu    (a CUDA box, needs oracle/_ref/libsolarref.so)
    ref_stage1_<name>.npz SHA-256 digests + per-voxel sample of the reference
                          viewshed stage (include/cuda/viewshed_stage.cuh:37-125):
                          CSR ids, ba-RLE bytes, shadow bitmap
    ref_annual_<name>.npz the reference API's annual irradiance (both pipelines)
    ref_stage1_blocks_dsm1024.npz
                          per block of 4096 voxels of the 1024 x 1024 city, SHA-256
                          digests of the reference viewshed stage's list lengths,
                          CSR ids, ba-RLE sizes and bytes and shadow bitmap, plus a
                          digest of the generated scene's arrays

  tiff   (this container: the reference tree and PIL)
    ref_dsm_tiff.json     the reference's test heightmap (test_data/dsm_heightmap.tiff:
                          tiled, Deflate, floating-point predictor) as decoded by PIL
                          (libtiff): shape, SHA-256 of the float32 heights, GeoTIFF tags

    python tests/golden/make_golden.py host
    python tests/golden/make_golden.py gpu [--out DIR]
    python tests/golden/make_golden.py gpu-large [--out DIR]
    python tests/golden/make_golden.py tiff
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from solargpu_b200 import inputs  # noqa: E402

SMALL = ("dsm64", "dsm160")


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def save_scene(name: str):
    s = inputs.make_scene(name)
    np.savez_compressed(os.path.join(HERE, f"scene_{name}.npz"), width=s.width, height=s.height,
                        **s.arrays())
    return s


def barle_lists(rng: np.random.Generator) -> list[np.ndarray]:
    """Id lists covering every width class, long runs (> 255), single-element
    outliers one class narrower (the optimiser's absorb rule) and empty lists."""
    out = [np.zeros(0, np.int32), np.array([1], np.int32), np.array([15], np.int32),
           np.array([16], np.int32), np.array([2 ** 31 - 1], np.int32),
           np.arange(1, 600, dtype=np.int32), np.arange(1, 2000, 3, dtype=np.int32)]
    for n in (2, 3, 5, 9, 17, 40, 145, 300, 700, 2592):
        for scale in (8, 200, 60000, 10_000_000, 2_000_000_000):
            ids = np.unique(rng.integers(1, scale + 2, size=n)).astype(np.int32)
            out.append(rng.permutation(ids))
    for _ in range(60):
        # mixed gaps: mostly small, some single large jumps
        gaps = rng.choice([1, 2, 7, 15, 16, 200, 255, 256, 70000, 20_000_000], size=rng.integers(2, 80),
                          p=[.3, .2, .1, .1, .05, .05, .05, .05, .05, .05])
        ids = np.cumsum(gaps)
        ids = ids[ids < 2 ** 31 - 1].astype(np.int32)
        out.append(rng.permutation(ids))
    return out


def host():
    if O.ref_host() is None:
        raise SystemExit("oracle/_ref/libref_host.so is missing (build oracle/ with the reference tree present)")
    rng = np.random.default_rng(2026)
    lists = barle_lists(rng)
    off = np.zeros(len(lists) + 1, np.int64)
    off[1:] = np.cumsum([len(x) for x in lists])
    ids = np.concatenate(lists).astype(np.int32)
    enc = [O.ref_barle_compress(x) for x in lists]
    boff = np.zeros(len(lists) + 1, np.int64)
    boff[1:] = np.cumsum([len(b) for b in enc])
    np.savez_compressed(os.path.join(HERE, "barle_golden.npz"), off=off, ids=ids, boff=boff,
                        bytes=np.frombuffer(b"".join(enc), np.uint8))
    for name in SMALL:
        s = save_scene(name)
        b = O.ref_sky_bins(s.sun)
        cfg = inputs.CONFIGS[name]
        ref_sun = O.ref_sun_positions(cfg.lon, cfg.lat, cfg.tz)
        np.savez_compressed(os.path.join(HERE, f"sky_{name}.npz"), ref_sun=ref_sun, full_to_dense=b["full_to_dense"],
                            sun_dense_idx=b["sun_dense_idx"], nudged=b["nudged"],
                            meta=np.array([b["hsize"], b["vsize"], b["vsize_full"], b["active"], b["words8"]]))
        H, W = s.height, s.width
        par, z, asp, sl, ta = O.ref_voxelize(s.grid.reshape(H, W))
        np.savez_compressed(os.path.join(HERE, f"voxel_{name}.npz"), parent=par, z=z, aspect=asp,
                            slope=sl, top_aspect=ta)
    print("host fixtures written to", HERE)


def gpu(out_dir: str):
    if O.ref_gpu() is None:
        raise SystemExit("oracle/_ref/libsolarref.so is missing")
    os.makedirs(out_dir, exist_ok=True)
    for name in SMALL:
        d = np.load(os.path.join(HERE, f"scene_{name}.npz"))
        s = inputs.scene_from_arrays(name, d, int(d["width"]), int(d["height"]))
        r = O.ref_stage1(s)
        counts = np.diff(r["csr_off"])
        rng = np.random.default_rng(7)
        sample = np.sort(rng.choice(s.num_total, size=min(64, s.num_total), replace=False))
        samp_ids = [r["csr_ids"][r["csr_off"][v]:r["csr_off"][v + 1]] for v in sample]
        samp_bytes = [r["barle"][r["barle_off"][v]:r["barle_off"][v + 1]] for v in sample]
        so = np.zeros(len(sample) + 1, np.int64)
        so[1:] = np.cumsum([len(x) for x in samp_ids])
        sb = np.zeros(len(sample) + 1, np.int64)
        sb[1:] = np.cumsum([len(x) for x in samp_bytes])
        np.savez_compressed(
            os.path.join(out_dir, f"ref_stage1_{name}.npz"),
            counts=counts.astype(np.int32), sha_ids=sha(r["csr_ids"].astype(np.int32)),
            sha_barle=sha(r["barle"]), sha_barle_off=sha(r["barle_off"].astype(np.int64)),
            sha_svf=sha(r["svf"]), svf_words8=r["svf"].shape[0],
            sample=sample, sample_off=so, sample_ids=np.concatenate(samp_ids).astype(np.int32),
            sample_boff=sb, sample_bytes=np.concatenate(samp_bytes).astype(np.uint8),
            svf=r["svf"] if s.num_total <= 20000 else np.zeros(0, np.uint8))
        unc = O.ref_irradiance(s, compressed=False)
        com = O.ref_irradiance(s, compressed=True)
        np.savez_compressed(os.path.join(out_dir, f"ref_annual_{name}.npz"), uncompressed=unc, compressed=com)
        print(name, "nnz", int(counts.sum()), "barle bytes", r["barle"].size)
    print("gpu fixtures written to", out_dir)


BLOCK = 4096


def scene_digest(s) -> str:
    h = hashlib.sha256()
    for a in (s.grid, s.pixel_parent, s.wall_z, s.slopes, s.aspects, s.sun, s.direct, s.diffuse):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def block_digests(off, ids, boff, barle, svf8, v0, v1) -> list[str]:
    """Digests of voxels [v0, v1): list lengths (int32), CSR ids (int32),
    ba-RLE sizes (int32), ba-RLE bytes, shadow bitmap in the reference layout
    (uint8 [words8][v1 - v0])."""
    return [sha(np.diff(off[v0:v1 + 1]).astype(np.int32)), sha(ids[off[v0]:off[v1]].astype(np.int32)),
            sha(np.diff(boff[v0:v1 + 1]).astype(np.int32)), sha(barle[boff[v0]:boff[v1]].astype(np.uint8)),
            sha(np.ascontiguousarray(svf8[:, v0:v1]))]


def gpu_large(out_dir: str, name: str = "dsm1024"):
    if O.ref_gpu() is None:
        raise SystemExit("oracle/_ref/libsolarref.so is missing")
    os.makedirs(out_dir, exist_ok=True)
    s = inputs.make_scene(name)
    r = O.ref_stage1(s)
    n = s.num_total
    dig = [block_digests(r["csr_off"], r["csr_ids"], r["barle_off"], r["barle"], r["svf"], v0, min(n, v0 + BLOCK))
           for v0 in range(0, n, BLOCK)]
    np.savez_compressed(os.path.join(out_dir, f"ref_stage1_blocks_{name}.npz"), block=BLOCK, num_total=n,
                        scene=scene_digest(s), digests=np.array(dig), nnz=int(r["csr_ids"].size),
                        barle_bytes=int(r["barle"].size), svf_words8=int(r["svf"].shape[0]))
    print(name, "blocks", len(dig), "nnz", r["csr_ids"].size, "barle bytes", r["barle"].size)


def tiff():
    import json
    from PIL import Image
    ref = os.environ.get("SOLARGPU_REFERENCE", "/root/reference")
    path = os.path.join(ref, "test_data", "dsm_heightmap.tiff")
    im = Image.open(path)
    a = np.array(im, dtype=np.float32)
    tags = im.tag_v2
    out = {"file": "test_data/dsm_heightmap.tiff", "shape": list(a.shape), "sha256_float32": sha(a),
           "min": float(a.min()), "max": float(a.max()),
           "pixel_scale": list(tags.get(33550, ())), "tiepoints": list(tags.get(33922, ())),
           "nodata": str(tags.get(42113, "")), "compression": int(tags.get(259, 1)),
           "predictor": int(tags.get(317, 1)), "tile": [int(tags.get(322, 0)), int(tags.get(323, 0))]}
    with open(os.path.join(HERE, "ref_dsm_tiff.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["host", "gpu", "gpu-large", "tiff"])
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if a.what == "host":
        host()
    elif a.what == "gpu":
        gpu(a.out)
    elif a.what == "tiff":
        tiff()
    else:
        gpu_large(a.out)
