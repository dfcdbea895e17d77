"""Test infrastructure (checker only): the reference CLI's own inputs through
both pipelines.

Reads a directory holding the reference's test data (dsm_heightmap.tiff,
tmy_direct.txt, tmy_diffuse.txt; test_data/ of the reference tree), builds
the inputs exactly as the reference CLI does (src/main.cpp:70-127: pixel size
from the GeoTIFF, lon 15.592, lat 46.543, UTC offset round(lon / 15)), and
compares, on the GPU:

  * this library's neighbor lists, ba-RLE streams and shadow words with the
    CPU oracle's and with the reference's own viewshed stage (bit-exact
    expected);
  * this library's annual irradiance (both list formats) with the reference
    pipeline's stock API (oracle/_ref/libsolarref.so, both entry points) and
    with the FP64 oracle on the same lists.

    python oracle/ref_data_check.py --data <dir with the reference test data>

Prints one JSON line.  Needs a GPU and oracle/_ref (built from the reference
sources by oracle/Makefile); the data directory is passed in because the
reference tree itself is not where the GPU runs.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    r = np.abs(a - b) / np.maximum(np.abs(b), 1.0)
    return {"max_rel": float(r.max()), "mean_rel": float(r.mean())}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--data", required=True)
    ap.add_argument("--lon", type=float, default=15.592)
    ap.add_argument("--lat", type=float, default=46.543)
    a = ap.parse_args(argv)
    import torch
    from conftest import device_arrays
    from oracle import oracle as O
    from solargpu_b200 import api, geotiff, inputs
    heights, meta = geotiff.read_tiff(os.path.join(a.data, "dsm_heightmap.tiff"))
    tz = int(round(a.lon / 15.0))
    direct = geotiff.read_tmy_series(os.path.join(a.data, "tmy_direct.txt"))
    diffuse = geotiff.read_tmy_series(os.path.join(a.data, "tmy_diffuse.txt"))
    s = inputs.scene_from_heightmap("dsm_heightmap.tiff", heights, float(meta.pixel_scale[0]), a.lon, a.lat, tz,
                                    direct, diffuse)
    res = {"input": "reference test_data: dsm_heightmap.tiff (%d x %d, %.2f-%.2f m) + TMY files" %
           (s.width, s.height, float(heights.min()), float(heights.max())),
           "voxels": s.num_total, "top_voxels": s.num_top, "lon": a.lon, "lat": a.lat, "tz": tz}
    off, ids, sh = O.trace(s, O.sky_bins(s.sun))
    fp64, _ = O.annual_fp64(s, sh, off, ids)
    d = device_arrays(s)
    with api.Context(0) as ctx:
        r = ctx.trace(s, d, neighbor_format=2)
        boff, bbytes = O.barle_encode_csr(off, ids)
        res["lists_vs_oracle"] = "bit-exact" if (np.array_equal(r["csr_off"], off) and np.array_equal(r["csr_ids"], ids)
                                                and np.array_equal(r["barle_off"], boff)
                                                and np.array_equal(r["barle"], bbytes)
                                                and np.array_equal(r["shadow"], sh)) else "DIFFERENT"
        rs = O.ref_stage1(s)
        res["lists_vs_reference_stage"] = "bit-exact" if (
            np.array_equal(r["csr_off"], rs["csr_off"]) and np.array_equal(r["csr_ids"], rs["csr_ids"])
            and np.array_equal(r["barle_off"], rs["barle_off"]) and np.array_equal(r["barle"], rs["barle"])
            and np.array_equal(r["shadow"], O.svf_to_words32(rs["svf"], r["shadow_words"]))) else "DIFFERENT"
        ours = {}
        for fmt, name in ((0, "CSR"), (1, "ba-RLE")):
            out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
            ctx.run_device(s, d, out, neighbor_format=fmt)
            torch.cuda.synchronize()
            ours[name] = out.cpu().numpy()
    ref = {"CSR": O.ref_irradiance(s, compressed=False), "ba-RLE": O.ref_irradiance(s, compressed=True)}
    for name in ("CSR", "ba-RLE"):
        res[name] = {"ours_vs_reference": rel(ours[name], ref[name]), "ours_vs_fp64": rel(ours[name], fp64),
                     "reference_vs_fp64": rel(ref[name], fp64)}
    print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
