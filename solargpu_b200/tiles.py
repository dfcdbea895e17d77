"""Many uneven tiles through the irradiance path, with an autotuner.

    python -m solargpu_b200.tiles [--tiles 32] [--seed 0] [--workers 2] [--tune] [--table tune.json]

The tile set: sides log-uniform in [128, 1024] cells (multiples of 16), the
1024 city's building and tree densities, a site per tile (latitude
U(35, 60), longitude U(-10, 30), time zone = round(lon / 15)) and its own
TMY seed; sun positions, sky bins and hour tables are computed per tile.
Tiles are generated on the host and uploaded once; each run is one
`solar_gpu_run_device` call (Stage 1 + the graph-captured hour-block loop).

Worker threads each own a context and a CUDA stream, so the small tiles of
one worker overlap the host-side set-up and launches of another (the ctypes
calls release the GIL).  `--batch` also runs all tiles through
solar_gpu_run_batch: Stage 1 and the list builds tile by tile, then the
hour-block loops of every tile as branches of one CUDA graph, launched once.  The autotuner times each candidate configuration
(list format x hour block x reflection kernel) on the first tile of a size
bucket (log2 of the voxel count), alone on the GPU before the workers start,
and reuses the fastest for the bucket; the table can be saved and reloaded
as JSON.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import threading
import time

import numpy as np

from . import inputs

CANDIDATES = (tuple(dict(neighbor_format=f, hour_block=b, group_size=g)
                    for f in (0, 1) for b in (128, 256) for g in (1, 64))
              + tuple(dict(neighbor_format=f, hour_block=256, group_size=128) for f in (0, 1)))
DEFAULT = dict(neighbor_format=0, hour_block=256, group_size=128)


def tile_configs(n: int = 32, seed: int = 0) -> list[inputs.DsmConfig]:
    """The seeded tile set (see the module docstring)."""
    rng = np.random.default_rng(seed)
    city = inputs.CONFIGS["dsm1024"]
    out = []
    for i in range(n):
        side = int(2.0 ** rng.uniform(7.0, 10.0)) // 16 * 16
        side = min(1024, max(128, side))
        area = (side / city.size) ** 2
        lat = float(rng.uniform(35.0, 60.0))
        lon = float(rng.uniform(-10.0, 30.0))
        out.append(inputs.DsmConfig(f"tile{i:02d}_{side}", side, max(1, round(city.n_buildings * area)),
                                    max(1, round(city.n_trees * area)), lat=round(lat, 4), lon=round(lon, 4),
                                    tz=int(round(lon / 15.0)), seed=100000 * (seed + 1) + i))
    return out


def size_bucket(scene) -> int:
    return int(round(math.log2(max(2, scene.num_total))))


class Autotuner:
    """Fastest candidate per size bucket, measured on the first tile seen."""

    def __init__(self, candidates=CANDIDATES, path: str | None = None):
        self.candidates = [dict(c) for c in candidates]
        self.path = path
        self.table: dict[int, dict] = {}
        self.trials: dict[int, list] = {}
        self.lock = threading.Lock()
        if path and os.path.exists(path):
            with open(path) as f:
                self.table = {int(k): v for k, v in json.load(f).items()}

    def choose(self, bucket: int, measure) -> dict:
        """measure(params) -> milliseconds; called for each candidate the
        first time a bucket is seen (measure may be None once every bucket
        in use has been tuned)."""
        with self.lock:
            if bucket in self.table:
                return self.table[bucket]
        trials = [(measure(c), c) for c in self.candidates]
        best = min(trials, key=lambda t: t[0])[1]
        with self.lock:
            self.table.setdefault(bucket, best)
            self.trials[bucket] = [(round(ms, 3), c) for ms, c in trials]
            if self.path:
                with open(self.path, "w") as f:
                    json.dump({str(k): v for k, v in self.table.items()}, f, indent=1)
            return self.table[bucket]


def _device_arrays(scene, dev):
    import torch
    wz = scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)
    return {"grid": torch.from_numpy(scene.grid).to(dev), "pixel_parent": torch.from_numpy(scene.pixel_parent).to(dev),
            "wall_z": torch.from_numpy(wz).to(dev), "slopes": torch.from_numpy(scene.slopes).to(dev),
            "aspects": torch.from_numpy(scene.aspects).to(dev)}


def run_tiles(scenes: list, params: dict | None = None, tuner: Autotuner | None = None, workers: int = 1,
              device: int = 0, accumulation: int = 1, keep_outputs: bool = False) -> dict:
    """Runs every scene once (after one untimed run per worker and
    configuration, which sizes the context's buffers).  Returns per-tile
    device times, the parameters used, the wall time of the timed pass and
    the aggregate voxel-hours/s."""
    import torch
    from . import api

    dev = torch.device("cuda", device)
    torch.cuda.set_device(dev)
    staged = [(s, _device_arrays(s, dev), torch.empty(s.num_total, dtype=torch.float32, device=dev)) for s in scenes]
    results: list = [None] * len(scenes)
    errors: list = []

    if tuner is not None:
        # Tuning runs first, alone on the GPU (one context, one stream), on
        # the first tile of each size bucket: the median of 3 timed runs of
        # each candidate after an untimed one.
        stream = torch.cuda.Stream(device=dev)
        with api.Context(device) as ctx:
            for s, d, out in staged:
                def measure(c):
                    ctx.run_device(s, d, out, stream=stream.cuda_stream, accumulation=accumulation, **c)
                    ms = []
                    for _ in range(3):
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record(stream)
                        ctx.run_device(s, d, out, stream=stream.cuda_stream, accumulation=accumulation, **c)
                        e1.record(stream)
                        e1.synchronize()
                        ms.append(e0.elapsed_time(e1))
                    return sorted(ms)[1]
                tuner.choose(size_bucket(s), measure)

    def run_one(ctx, stream, i, timed):
        s, d, out = staged[i]
        p = dict(params or DEFAULT)
        if tuner is not None:
            p = tuner.choose(size_bucket(s), None)
        if not timed:
            ctx.run_device(s, d, out, stream=stream.cuda_stream, accumulation=accumulation, **p)
            return
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.run_device(s, d, out, stream=stream.cuda_stream, accumulation=accumulation, **p)
        e1.record(stream)
        e1.synchronize()
        hd = int(((s.sun[:, 1] - np.float32(1e-8)) >= 1.0).sum())
        results[i] = {"tile": s.name, "voxels": s.num_total, "daylight_hours": hd, "ms": e0.elapsed_time(e1),
                      "params": p}
        if keep_outputs:
            results[i]["out"] = out.cpu().numpy()

    warm_done = threading.Barrier(workers + 1)
    start = threading.Barrier(workers + 1)

    def worker(w):
        mine = list(range(w, len(scenes), workers))
        ctx = stream = None
        try:
            torch.cuda.set_device(dev)
            stream = torch.cuda.Stream(device=dev)
            ctx = api.Context(device)
            for i in mine:              # warm: buffers sized, autotuner trials
                run_one(ctx, stream, i, False)
        except Exception as e:          # reported after the join
            errors.append(e)
        warm_done.wait()
        start.wait()
        try:
            if not errors:
                for i in mine:
                    run_one(ctx, stream, i, True)
        except Exception as e:
            errors.append(e)
        finally:
            if ctx is not None:
                ctx.close()

    threads = [threading.Thread(target=worker, args=(w,)) for w in range(workers)]
    for t in threads:
        t.start()
    warm_done.wait()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    start.wait()
    for t in threads:
        t.join()
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t0
    if errors:
        raise errors[0]
    vh = float(sum(r["voxels"] * r["daylight_hours"] for r in results))
    return {"tiles": results, "wall_s": wall, "voxel_hours": vh, "voxel_hours_per_s": vh / wall,
            "sum_tile_ms": sum(r["ms"] for r in results)}


def run_tiles_batched(scenes: list, params: dict | None = None, tuner: Autotuner | None = None, device: int = 0,
                      accumulation: int = 1, runs: int = 2, keep_outputs: bool = False) -> dict:
    """Every tile in one batch (solar_gpu_run_batch): one context per tile,
    Stage 1 and the list builds tile by tile, then all hour-block loops as
    branches of one CUDA graph.  One untimed batch sizes the buffers; the
    median of `runs` timed batches (CUDA events around the call) is
    reported.  With a tuner, each tile runs the configuration its size bucket
    was tuned to (tune first, e.g. with run_tiles)."""
    import torch
    from . import api

    dev = torch.device("cuda", device)
    torch.cuda.set_device(dev)
    devs = [_device_arrays(s, dev) for s in scenes]
    outs = [torch.empty(s.num_total, dtype=torch.float32, device=dev) for s in scenes]
    per_tile = []
    for s in scenes:
        p = dict(params or DEFAULT)
        if tuner is not None and size_bucket(s) in tuner.table:
            p = dict(tuner.table[size_bucket(s)])
        p["accumulation"] = accumulation
        per_tile.append(p)
    ctxs = [api.Context(device) for _ in scenes]
    stream = torch.cuda.Stream(device=dev)
    try:
        api.run_batch(ctxs, scenes, devs, outs, stream=stream.cuda_stream, per_tile=per_tile)
        ms = []
        for _ in range(max(1, runs)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            e0.record(stream)
            api.run_batch(ctxs, scenes, devs, outs, stream=stream.cuda_stream, per_tile=per_tile)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    finally:
        for c in ctxs:
            c.close()
    vh = float(sum(s.num_total * int(((s.sun[:, 1] - np.float32(1e-8)) >= 1.0).sum()) for s in scenes))
    t = sorted(ms)[len(ms) // 2]
    r = {"batch_ms": [round(x, 2) for x in ms], "median_ms": round(t, 2), "voxel_hours": vh,
         "voxel_hours_per_s": vh / (t / 1e3), "params": per_tile}
    if keep_outputs:
        r["outs"] = [o.cpu().numpy() for o in outs]
    return r


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--tiles", type=int, default=32)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--workers", type=int, default=2)
    ap.add_argument("--tune", action="store_true", help="autotune per size bucket (else the default path)")
    ap.add_argument("--table", default=None, help="autotuner table (JSON) to load and update")
    ap.add_argument("--batch", action="store_true",
                    help="also run every tile in one batch (one CUDA graph over all hour loops)")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    scenes = [inputs.make_scene(c) for c in tile_configs(a.tiles, a.seed)]
    gen_s = time.perf_counter() - t0
    tuner = Autotuner(path=a.table) if a.tune else None
    r = run_tiles(scenes, tuner=tuner, workers=a.workers)
    r["generate_s"] = gen_s
    r["workers"] = a.workers
    if tuner is not None:
        r["autotuner"] = {str(k): {"chosen": v, "trials_ms": tuner.trials.get(k)} for k, v in tuner.table.items()}
    if a.batch:
        b = run_tiles_batched(scenes, tuner=tuner)
        r["batched"] = {k: v for k, v in b.items() if k != "params"}
    print(json.dumps(r))
    return 0


if __name__ == "__main__":
    sys.exit(main())
