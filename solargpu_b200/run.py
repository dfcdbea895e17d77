"""Command-line runner: the annual irradiance path on a GeoTIFF heightmap or a named synthetic workload.

    python -m solargpu_b200.run --workload dsm1024 [--format 0] [--hour-block 256]
                                [--group-size 128] [--accumulation 1] [--runs 2] [--out file.npy|file.tiff]
                                [--dump file_voxels.bin] [--compare-accumulation]
    python -m solargpu_b200.run --dsm heightmap.tiff [--lon 15.592] [--lat 46.543] [--tz N]
                                [--direct tmy_direct.txt --diffuse tmy_diffuse.txt] [--out out.tiff]

Plays the role of the reference CLI (src/main.cpp): reads the heightmap
(--dsm, a single-band float32 GeoTIFF; pixel size from its pixel-scale tag)
or builds a seeded synthetic DSM, voxelizes it, computes the sun series and
reads or generates the TMY series, runs the CUDA pipeline `--runs` times on
device-resident inputs and prints the stage and kernel-group times of the
last run; --out writes the top voxels' raster (a GeoTIFF with the input's
georeferencing when the name ends in .tif/.tiff, else .npy) and --dump the
reference's voxel dump (solargpu_b200/outputs.py).  Also the profiling driver
(run it under ncu with -k/-s/-c filters).  --compare-accumulation runs the
three accumulation modes (FP64 block sums, Kahan FP32, plain FP32) on the
same scene and reports the relative differences of the last two from the
first, with each mode's time.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workload", default="dsm1024")
    ap.add_argument("--dsm", default=None, help="GeoTIFF heightmap (replaces --workload)")
    ap.add_argument("--lon", type=float, default=15.592)
    ap.add_argument("--lat", type=float, default=46.543)
    ap.add_argument("--tz", type=int, default=None, help="UTC offset of the TMY hours (default: round(lon / 15))")
    ap.add_argument("--direct", default=None, help="hourly direct irradiance, 8760 values (default: synthetic)")
    ap.add_argument("--diffuse", default=None, help="hourly diffuse irradiance, 8760 values (default: synthetic)")
    ap.add_argument("--format", type=int, default=0, help="0 = CSR, 1 = ba-RLE")
    ap.add_argument("--hour-block", type=int, default=256)
    ap.add_argument("--group-size", type=int, default=128)
    ap.add_argument("--accumulation", type=int, default=1)
    ap.add_argument("--chunk-voxels", type=int, default=0)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--out", default=None, help="write the top voxels' annual irradiance raster (float32 .npy)")
    ap.add_argument("--dump", default=None, help="write the voxel dump of the reference CLI (x, y, z, irradiance)")
    ap.add_argument("--compare-accumulation", action="store_true")
    a = ap.parse_args(argv)

    import torch
    from solargpu_b200 import api, inputs

    meta = None
    if a.dsm:
        from solargpu_b200 import geotiff
        heights, meta = geotiff.read_tiff(a.dsm)
        if len(meta.pixel_scale) < 2:
            raise SystemExit(f"TIFF {a.dsm} missing GeoTIFF pixel-scale tag")
        tz = a.tz if a.tz is not None else int(round(a.lon / 15.0))
        direct = geotiff.read_tmy_series(a.direct) if a.direct else None
        diffuse = geotiff.read_tmy_series(a.diffuse) if a.diffuse else None
        s = inputs.scene_from_heightmap(os.path.basename(a.dsm), heights, float(meta.pixel_scale[0]), a.lon, a.lat,
                                        tz, direct, diffuse)
    else:
        s = inputs.make_scene(a.workload)
    dev = torch.device("cuda:0")
    d = {"grid": torch.from_numpy(s.grid).to(dev), "pixel_parent": torch.from_numpy(s.pixel_parent).to(dev),
         "wall_z": torch.from_numpy(s.wall_z if s.wall_z.size else np.zeros(1, np.float32)).to(dev),
         "slopes": torch.from_numpy(s.slopes).to(dev), "aspects": torch.from_numpy(s.aspects).to(dev)}
    out = torch.zeros(s.num_total, dtype=torch.float32, device=dev)
    if a.compare_accumulation:
        res, ms = {}, {}
        with api.Context(0) as ctx:
            for acc in (0, 1, 2):
                ctx.run_device(s, d, out, neighbor_format=a.format, hour_block=a.hour_block,
                               group_size=a.group_size, accumulation=acc, chunk_voxels=a.chunk_voxels,
                               use_graph=1, time_kernels=0)
                torch.cuda.synchronize()
                ms[acc] = round(ctx.timings()[3], 1)
                res[acc] = out.double().clone()
        ref = res[0]
        den = ref.abs().clamp_min(1.0)
        cmp = {}
        for acc, name in ((1, "kahan_fp32"), (2, "plain_fp32")):
            r = (res[acc] - ref).abs() / den
            cmp[name] = {"max_rel_vs_fp64_sums": float(r.max()), "mean_rel_vs_fp64_sums": float(r.mean())}
        print(json.dumps({"workload": a.workload, "voxels": s.num_total, "top_voxels": s.num_top,
                          "total_ms": {"fp64_sums": ms[0], "kahan_fp32": ms[1], "plain_fp32": ms[2]},
                          "accumulation": cmp}))
        return 0
    with api.Context(0) as ctx:
        for _ in range(max(1, a.runs)):
            ctx.run_device(s, d, out, neighbor_format=a.format, hour_block=a.hour_block,
                           group_size=a.group_size, accumulation=a.accumulation,
                           chunk_voxels=a.chunk_voxels, use_graph=0, time_kernels=1)
            torch.cuda.synchronize()
        t = ctx.timings()
        kt = {k: round(v[0], 3) for k, v in ctx.kernel_times().items() if v[1]}
    print(json.dumps({"workload": a.dsm or a.workload, "voxels": s.num_total, "top_voxels": s.num_top,
                      "stage_ms": {"setup": round(t[0], 3), "stage1": round(t[1], 3), "stage23": round(t[2], 3),
                                   "total": round(t[3], 3)}, "kernel_group_ms": kt}))
    from solargpu_b200 import outputs
    if a.out:
        if a.out.lower().endswith((".tif", ".tiff")):
            outputs.write_geotiff(a.out, s, out.cpu().numpy(), meta)
        else:
            outputs.write_raster(a.out, s, out.cpu().numpy())
    if a.dump:
        outputs.write_voxel_dump(a.dump, s, out.cpu().numpy())
    return 0


if __name__ == "__main__":
    sys.exit(main())
