"""Benchmark: annual voxel-hours/s of the whole irradiance path on B200.

One step = one complete annual run on the resident scene: Stage 1 (DDA
viewshed tracer, neighbor lists, shadow bits) and Stage 2/3 (solar +
hour-block reflection + accumulation over all daylight hours).
voxel-hours = voxels x daylight hours.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica of the workload (the
path shards by DSM tile with no exchange), value = all ranks' voxel-hours /
the slowest rank's time.  `--impl reference` times the reference's own
implementation (its CUDA pipeline rebuilt from source for sm_100a, called
through its stock API) on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "annual voxel-hours/s on 1 B200 vs plain per-hour path at ≤1e-4 rel err"
UNIT = "voxel-hours/s"
N_DIRS = 2592      # traced directions per voxel: 72 azimuth x 36 elevation bins of 5 degrees
FMT_NAMES = {0: "CSR", 1: "ba-RLE"}
ACC_NAMES = {0: "fp32 block sums + fp64 annual", 1: "kahan-compensated fp32", 2: "plain fp32"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="dsm1024")
    ap.add_argument("--format", type=int, default=0, help="0 = CSR, 1 = ba-RLE")
    ap.add_argument("--hour-block", type=int, default=256)
    ap.add_argument("--accumulation", type=int, default=1)
    ap.add_argument("--group-size", type=int, default=128)
    ap.add_argument("--ref-workload", default=None,
                    help="reference arm: workload timed per step (default: the arm's own workload; its "
                         "uncompressed path takes 24 s per annual run of dsm1024, the compressed one ~6 min)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-hour comparison run")
    ap.add_argument("--no-check", action="store_true", help="skip the FP64 error check")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-config3", action="store_true",
                    help="skip the 4096 x 4096 city block (config3 key: default path, plain per-hour path, "
                         "accumulation variants, sampled FP64 oracle and list parity)")
    ap.add_argument("--config3-workload", default="dsm4096", help="workload of the config3 block")
    ap.add_argument("--no-config3-plain", action="store_true",
                    help="config3 block without its plain per-hour run (about 5 minutes at 4096 x 4096)")
    ap.add_argument("--no-config4", action="store_true",
                    help="skip the 32-tile block (config4 key: one batched graph against tile-by-tile runs)")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons.  Started
    before the warm-up (nvidia-smi's own start-up slows the GPU's host side
    for a few hundred ms); mark() opens the timed region, stop() closes it and
    summarises the samples taken in between."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.first = 0

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_ready(self, samples: int = 3, timeout_s: float = 5.0):
        """Returns once nvidia-smi has delivered a few samples (past its start-up)."""
        t0 = time.perf_counter()
        while self.proc is not None and len(self.lines) < samples and time.perf_counter() - t0 < timeout_s:
            time.sleep(0.05)

    def mark(self):
        self.first = len(self.lines)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        timed = self.lines[self.first:] or self.lines
        for ln in timed:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- helpers

def dist_setup(args=None, backend: str | None = None):
    """One process per GPU (torchrun env); NCCL on GPUs, gloo without (tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x: float, device) -> float:
    """The slowest rank's time (every rank gets it)."""
    if pg is None:
        return x
    import torch
    if pg.get_backend() == "gloo":
        device = "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: float, steps: int, slowest_ms: float) -> float:
    """Whole-job rate: every rank's units over the slowest rank's time."""
    return world * units_per_rank * steps / (slowest_ms / 1e3)


_PINNED = []


def pinned_copy(a: np.ndarray) -> np.ndarray:
    """A copy of `a` in page-locked host memory (kept alive for the run)."""
    import torch
    t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
    _PINNED.append(t)
    out = t.numpy()
    out[...] = a
    return out


def workload_desc(scene, name: str) -> str:
    from solargpu_b200 import inputs
    c = inputs.CONFIGS[name]
    return (f"{name}: seeded synthetic DSM {c.size}x{c.size} @1 m, {c.n_buildings} buildings "
            f"({c.side_min}-{c.side_max} m, roofs {c.roof_min:g}-{c.roof_max:g} m), {c.n_trees} Gaussian trees, "
            f"{scene.num_top} top + {scene.num_total - scene.num_top} wall voxels, "
            f"lat {c.lat} lon {c.lon} tz +{c.tz}, synthetic TMY")


def roofline_bytes(scene, ctx_sizes, fmt, B, acc, V, entries, staged_rows=0) -> float:
    """Algorithmic HBM bytes of one hour-block reflection launch, gathered
    slab rows counted once (as cache hits): the streamed lists, per voxel the
    visiting-order index and accumulator read/write, and one read of the
    block's slab.
      V = 0: CSR ids or ba-RLE bytes + offsets; geometry and shadow words per
             voxel; slab rows of the top cells.
      V = 1, 2, 4, 8: entries of one cell id + V weights, group offsets; the
             slab has a row for every voxel (its own term).
      V = 64 (tiles): merged entries of a 2-byte row index + the 4 weights of
             a voxel quad, the groups' union cell ids and chunk tables (80 B
             per chunk of 80 rows, ~1 B per staged row), offsets; slab rows of
             every voxel.
      V = 128 (tensor cores): entries of 8 bytes (W-tile offset, fp16 hi and
             lo) per nonzero weight, the union cell id of every staged row,
             16 B of chunk offsets per 64 rows; per voxel the visiting-order
             index, scale, normal, shadow words and accumulator; the fp16
             slab of the top cells read once."""
    csr_entries, barle_bytes, words32 = ctx_sizes
    N, T = scene.num_total, scene.num_top
    acc_b = 16 if acc in (0, 1) else 8
    if V == 128:
        lists = entries * 8 + staged_rows * 4 + (staged_rows // 64) * 16 + 8 * (N + 1)
        return float(lists + N * (4 + 4 + 16 + 4 * words32 + acc_b) + T * B * 2)
    if V == 0:
        lists = (barle_bytes if fmt == 1 else 4 * csr_entries) + 8 * (N + 1)
        return float(lists + N * (4 + 32 + 4 * words32 + acc_b) + T * B * 4)
    if V >= 64:
        lists = entries * 18 + staged_rows * 5 + 8 * (N + 1)
    else:
        lists = entries * (4 + 4 * V) + 8 * (N // V + 2)
    return float(lists + N * (4 + acc_b) + N * B * 4)


# ---------------------------------------------------------------- sampled parity

def sample_ranges(scene, seed: int, n_top: int = 12, n_wall: int = 8, length: int = 1000):
    """Contiguous voxel ranges for the sampled checks: n_top ranges of top
    voxels (raster rows) and n_wall of wall voxels, `length` voxels each,
    disjoint.  Contiguous ranges keep the set of top cells their lists name
    small enough to trace on the host.  Returns (ranges, voxel ids)."""
    rng = np.random.default_rng(seed)
    T, N = scene.num_top, scene.num_total

    def pick(lo, hi, k):
        slots = (hi - lo) // length
        if slots <= k:
            return [(lo, hi)] if hi > lo else []
        starts = np.sort(rng.choice(slots, size=k, replace=False)) * length + lo
        return [(int(a), int(a + length)) for a in starts]

    ranges = pick(0, T, n_top) + pick(T, N, n_wall)
    return ranges, np.concatenate([np.arange(a, b, dtype=np.int32) for a, b in ranges])


def gpu_sample_lists(ranges, get) -> dict:
    """Concatenates the GPU's Stage 1 products of the sampled ranges; get(a, b)
    returns them for voxels [a, b) with offsets from 0 (Context.trace_range)."""
    parts = [get(a, b) for a, b in ranges]
    res = {"shadow": np.concatenate([g["shadow"] for g in parts])}
    for off_key, dat_key in (("csr_off", "csr_ids"), ("barle_off", "barle")):
        if off_key in parts[0]:
            offs, dat, base = [np.zeros(1, np.int64)], [], 0
            for g in parts:
                offs.append(g[off_key][1:] + base)
                dat.append(g[dat_key])
                base += int(g[off_key][-1])
            res[off_key], res[dat_key] = np.concatenate(offs), np.concatenate(dat)
    return res


def lists_vs_reference(O, scene, r: dict) -> dict:
    """Every voxel's CSR ids, ba-RLE bytes and shadow bits against the
    reference's own viewshed stage (include/cuda/viewshed_stage.cuh:37-125 with
    src/cuda/kernels/viewshed_kernels.cu:7-59, rebuilt from its sources for
    sm_100a), run after the timed region.  Never raises: a failure is
    recorded in the key."""
    try:
        if O.ref_gpu() is None:
            return {"result": "unavailable", "why": "reference CUDA pipeline not built (oracle/_ref)"}
        with quiet_stdout():   # the reference stage prints its chunking from C++
            ref = O.ref_stage1(scene)
        res = {"voxels": int(scene.num_total), "neighbor_ids": int(r["csr_off"][-1]),
               "reference": "the reference's viewshed stage rebuilt for sm_100a from its sources"}
        first = None
        if not np.array_equal(r["csr_off"], ref["csr_off"]):
            first = int(np.flatnonzero(np.diff(r["csr_off"]) != np.diff(ref["csr_off"]))[0])
        elif not np.array_equal(r["csr_ids"], ref["csr_ids"]):
            k = int(np.flatnonzero(r["csr_ids"] != ref["csr_ids"])[0])
            first = int(np.searchsorted(r["csr_off"], k, side="right") - 1)
        elif not np.array_equal(r["barle_off"], ref["barle_off"]):
            first = int(np.flatnonzero(np.diff(r["barle_off"]) != np.diff(ref["barle_off"]))[0])
        elif not np.array_equal(r["barle"], ref["barle"]):
            k = int(np.flatnonzero(r["barle"] != ref["barle"])[0])
            first = int(np.searchsorted(r["barle_off"], k, side="right") - 1)
        else:
            sh = O.svf_to_words32(ref["svf"], r["shadow_words"])
            if not np.array_equal(r["shadow"], sh):
                first = int(np.flatnonzero((r["shadow"] != sh).any(axis=1))[0])
        res["result"] = "bit-exact" if first is None else "DIFFERENT"
        if first is not None:
            res["first_differing_voxel"] = first
        return res
    except Exception as e:   # a checker, not the measurement: keep the line
        return {"result": "unavailable", "why": f"{type(e).__name__}: {e}"[:300]}


def list_parity(O, orc, gs: dict, cell_shadow_gpu: np.ndarray, smp: np.ndarray) -> dict:
    """Bit-exact comparison of the GPU's neighbor lists (CSR ids, ba-RLE bytes)
    and shadow words with the oracle's own traces of the same voxels, and of
    the shadow words of every top cell those lists name."""
    res = {"voxels_checked": int(smp.size), "cells_checked": int(orc["cells"].size),
           "oracle": "CPU restatement of the reference DDA (pinned to the reference kernel's own output)"}
    first = None

    def per_voxel(goff, gdat, ooff, odat):
        nonlocal first
        if np.array_equal(goff, ooff) and np.array_equal(gdat, odat):
            return 0
        bad = 0
        for k in range(smp.size):
            if not np.array_equal(gdat[goff[k]:goff[k + 1]], odat[ooff[k]:ooff[k + 1]]):
                bad += 1
                first = int(smp[k]) if first is None else first
        return bad

    if "csr_off" in gs:
        res["csr_mismatched_voxels"] = per_voxel(gs["csr_off"], gs["csr_ids"], orc["off"], orc["ids"])
    if "barle_off" in gs:
        boff, b = O.barle_encode_csr(orc["off"], orc["ids"])
        res["barle_mismatched_voxels"] = per_voxel(gs["barle_off"], gs["barle"], boff, b)
    bad_sh = np.nonzero((gs["shadow"] != orc["shadow"]).any(axis=1))[0]
    res["shadow_mismatched_voxels"] = int(bad_sh.size)
    if bad_sh.size and first is None:
        first = int(smp[bad_sh[0]])
    res["cell_shadow_mismatched"] = int((cell_shadow_gpu != orc["cell_shadow"]).any(axis=1).sum())
    clean = all(v == 0 for k, v in res.items() if k.endswith("mismatched_voxels") or k == "cell_shadow_mismatched")
    res["result"] = "bit-exact" if clean else f"mismatch (first differing voxel {first})"
    return res


def hours_of(scene) -> int:
    """Daylight hours the path runs (nudged altitude >= 1 deg)."""
    return int(((scene.sun[:, 1] - np.float32(1e-8)) >= 1.0).sum())


def run_config3(args, ctx, dev, stream, flush) -> dict:
    """The 4096 x 4096 city: the hour-block path (ba-RLE lists, the config's
    format, and CSR), the plain per-hour path once, the three accumulation
    variants, and a sampled check against the FP64 oracle on oracle-built
    lists (the oracle works on the host cores while the GPU runs)."""
    import torch
    from oracle import oracle as O
    from solargpu_b200 import api, inputs
    t0 = time.perf_counter()
    sc = inputs.make_scene(args.config3_workload)
    gen_s = time.perf_counter() - t0
    N, T = sc.num_total, sc.num_top
    Hd = hours_of(sc)
    units = float(N) * Hd
    d = {"grid": torch.from_numpy(sc.grid).to(dev), "pixel_parent": torch.from_numpy(sc.pixel_parent).to(dev),
         "wall_z": torch.from_numpy(sc.wall_z).to(dev), "slopes": torch.from_numpy(sc.slopes).to(dev),
         "aspects": torch.from_numpy(sc.aspects).to(dev)}
    out = torch.empty(N, dtype=torch.float32, device=dev)
    ranges, smp = sample_ranges(sc, seed=3)
    box = {}

    def oracle_side():
        try:
            box["orc"] = O.sample_reference(sc, smp)
        except Exception as e:   # reported in the key, never hidden
            box["err"] = repr(e)

    th = threading.Thread(target=oracle_side, daemon=True)
    th.start()

    def timed(opts, runs):
        ms, kt = [], {}
        for _ in range(runs):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.run_device(sc, d, out, stream=stream.cuda_stream, **opts)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(e0.elapsed_time(e1))
            if opts.get("time_kernels"):
                for g, (t, n) in ctx.kernel_times().items():
                    kt[g] = kt.get(g, 0.0) + t / runs
        return ms, kt

    base = dict(hour_block=256, accumulation=api.ACC_KAHAN, group_size=args.group_size, use_graph=0, time_kernels=1)
    res = {"workload": workload_desc(sc, args.config3_workload), "voxels": N, "daylight_hours": Hd,
           "host_generation_s": round(gen_s, 2),
           "reference": "unavailable at this size: the reference pipeline's int32 CSR / ba-RLE offsets "
                        "(src/cuda/gpu_irradiance_uncompressed.cu:79, gpu_irradiance_compressed.cu:81) overflow "
                        "above 2^31 entries, and this scene has more neighbor ids than that"}
    paths = {}
    for fmt in (api.BARLE, api.CSR):
        opts = dict(base, neighbor_format=fmt)
        ctx.run_device(sc, d, out, stream=stream.cuda_stream, **opts)   # warm-up (buffers, tables)
        torch.cuda.synchronize(dev)
        ms, kt = timed(opts, 2)
        paths[FMT_NAMES[fmt]] = {"ms_per_run": [round(x, 1) for x in ms],
                                 "value": units / (sum(ms) / len(ms) / 1e3),
                                 "stage_ms": {g: round(v, 1) for g, v in kt.items()}}
        if fmt == api.BARLE:
            kahan = out.cpu().numpy().astype(np.float64)
    res["hour_block_path"] = paths
    # accumulation variants on ba-RLE lists (kahan from the timed runs)
    accs = {api.ACC_KAHAN: kahan}
    for acc in (api.ACC_FP64, api.ACC_FP32):
        ctx.run_device(sc, d, out, stream=stream.cuda_stream, **dict(base, neighbor_format=api.BARLE,
                                                                    accumulation=acc, time_kernels=0))
        torch.cuda.synchronize(dev)
        accs[acc] = out.cpu().numpy().astype(np.float64)
    if not args.no_config3_plain:
        popts = dict(neighbor_format=api.CSR, hour_block=1, accumulation=api.ACC_FP32, use_graph=0, time_kernels=0)
        ms, _ = timed(popts, 1)
        res["plain_per_hour"] = {"ms_per_run": round(ms[0], 1), "value": units / (ms[0] / 1e3),
                                 "config": "hour_block 1 on CSR lists (one solar + one reflection launch per "
                                           "daylight hour), plain fp32; one timed run, cold (no warm-up: a run "
                                           "takes minutes)",
                                 "speedup_of_hour_block_path": {k: round(ms[0] / (sum(p["ms_per_run"]) / len(p["ms_per_run"])), 2)
                                                                for k, p in paths.items()},
                                 "target": ">= 5x"}
    # Stage 1 alone keeps both list formats on the device (a full run of a
    # scene this large releases them to make room for the hour loop)
    ctx.stage1(sc, d, neighbor_format=2, stream=stream.cuda_stream)
    gs = gpu_sample_lists(ranges, lambda a, b: ctx.trace_range(a, b, csr=True, barle=True))
    cell_sh = ctx.trace_range(0, T, csr=False)["shadow"]
    ctx.release()
    th.join()
    if "orc" not in box:
        res["oracle_error"] = box.get("err", "oracle sample did not finish")
        return res
    orc = box["orc"]
    res["list_parity"] = list_parity(O, orc, gs, cell_sh[orc["cells"]], smp)
    errs = {}
    for acc, o in accs.items():
        rel = np.abs(o[smp] - orc["annual"]) / np.maximum(np.abs(orc["annual"]), 1.0)
        errs[ACC_NAMES[acc]] = {"max_rel": float(rel.max()), "mean_rel": float(rel.mean())}
    res["error_vs_fp64_oracle"] = {"variants": errs, "voxels": int(smp.size),
                                   "sample": f"{len(ranges)} contiguous ranges of 1000 voxels (12 of top voxels, "
                                             f"8 of wall voxels), seeded",
                                   "oracle": "FP64 annual-sum oracle on oracle-built lists and shadow words: the "
                                             "sample's own traces and the traces of all "
                                             f"{orc['cells'].size} top cells its lists name",
                                   "oracle_host_s": round(orc["trace_s"] + orc["irradiance_s"], 1),
                                   "tolerance": 1e-4}
    return res


def run_config4(args) -> dict:
    """32 seeded uneven tiles (sides log-uniform in 128-1024, a site and TMY
    per tile): every tile in one batch (solar_gpu_run_batch: the hour loops
    of all tiles as branches of one CUDA graph) against the same tiles run one
    by one on one context and stream, both on the default path."""
    import torch
    from solargpu_b200 import inputs, tiles
    t0 = time.perf_counter()
    scenes = [inputs.make_scene(c) for c in tiles.tile_configs(32, seed=0)]
    gen_s = time.perf_counter() - t0
    one = tiles.run_tiles(scenes, workers=1)
    batch = tiles.run_tiles_batched(scenes, runs=3)
    torch.cuda.synchronize()
    return {"tiles": len(scenes), "voxels": int(sum(s.num_total for s in scenes)),
            "host_generation_s": round(gen_s, 2),
            "tile_by_tile": {"wall_ms": round(one["wall_s"] * 1e3, 1), "voxel_hours_per_s": one["voxel_hours_per_s"],
                             "how": "one context and stream, solar_gpu_run_device per tile (graph-captured hour "
                                    "loop each), wall clock around the pass"},
            "batched": {"ms": batch["batch_ms"], "median_ms": batch["median_ms"],
                        "voxel_hours_per_s": batch["voxel_hours_per_s"],
                        "how": "solar_gpu_run_batch: Stage 1 and list builds tile by tile, then every tile's "
                               "hour loop as a branch of one CUDA graph; CUDA events around the call, median of 3"},
            "speedup": round(one["wall_s"] * 1e3 / batch["median_ms"], 3)}


# ---------------------------------------------------------------- our arm

def run_ours(args, world, rank, local, pg):
    import torch
    from solargpu_b200 import api, inputs

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scene = inputs.make_scene(args.workload)
    N, T = scene.num_total, scene.num_top
    d = {
        "grid": torch.from_numpy(scene.grid).to(dev),
        "pixel_parent": torch.from_numpy(scene.pixel_parent).to(dev),
        "wall_z": torch.from_numpy(scene.wall_z).to(dev),
        "slopes": torch.from_numpy(scene.slopes).to(dev),
        "aspects": torch.from_numpy(scene.aspects).to(dev),
    }
    out = torch.empty(N, dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2
    stream = torch.cuda.current_stream(dev)
    ctx = api.Context(local)
    opts = dict(neighbor_format=args.format, hour_block=args.hour_block, accumulation=args.accumulation,
                group_size=args.group_size, use_graph=0, time_kernels=1)

    def step():
        ctx.run_device(scene, d, out, stream=stream.cuda_stream, **opts)

    sampler = ClockSampler(local)
    sampler.start()
    sampler.wait_ready()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    # ---- timed region
    sampler.mark()
    barrier(pg)
    torch.cuda.synchronize(dev)
    evs = []
    ktimes = {}
    launches = 0
    for _ in range(args.steps):
        flush.zero_()                       # untimed L2 flush between steps
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        evs.append((e0, e1))
        for g, (ms, n) in ctx.kernel_times().items():
            a = ktimes.setdefault(g, [0.0, 0])
            a[0] += ms
            a[1] += n
        launches += ctx.launches()
    torch.cuda.synchronize(dev)
    barrier(pg)
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(pg, sum(step_ms), dev)
    import ctypes as C
    ne, nb = C.c_longlong(), C.c_longlong()
    w, a_, n_ = C.c_int(), C.c_int(), C.c_int()
    api.lib().solar_gpu_trace_sizes(ctx.h, C.byref(ne), C.byref(nb), C.byref(w), C.byref(a_), C.byref(n_))
    Hd = int(((scene.sun[:, 1] - np.float32(1e-8)) >= 1.0).sum())
    units = float(N) * Hd
    value = aggregate_rate(world, units, args.steps, total_ms)
    ms_per_step = total_ms / args.steps

    # ---- dominant kernel roofline (live events over the timed region)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dom = max(ktimes.items(), key=lambda kv: kv[1][0])
    refl_ms, refl_n = ktimes.get("reflect", (0.0, 0))
    B = args.hour_block
    V = args.group_size
    entries = ctx.reflection_entries()
    staged = ctx.staged_rows()
    alg = roofline_bytes(scene, (ne.value, nb.value, w.value), args.format, B, args.accumulation, V, entries, staged)
    per_launch_ms = refl_ms / max(1, refl_n)
    achieved = alg / (per_launch_ms / 1e3) / 1e9 if per_launch_ms > 0 else 0.0
    # slab bytes delivered to the arithmetic per launch: the fp16 union rows
    # the tensor-core kernel stages into shared memory, else one row of B
    # floats per entry (through L1, or from shared memory for the tile kernel)
    gathered = float(staged) * B * 2 if V == 128 else float(entries if V >= 1 else ne.value) * B * 4
    # DRAM bytes per launch come from an ncu capture of this kernel and
    # workload (a profiler run cannot be a timed run); the file is named in
    # the line so that a stale figure can be told from a live one.
    traffic = None
    traffic_src = None
    kname = ("reflect_mma" if V == 128 else "reflect_tile" if V >= 64 else "reflect_group" if V >= 1
             else "reflect_block")
    prof = os.path.join("profiles", f"{kname}_{args.workload}_{FMT_NAMES[args.format].replace('-', '').lower()}_b{B}_v{V}.md")
    if os.path.exists(os.path.join(ROOT, prof)):
        for ln in open(os.path.join(ROOT, prof)):
            if ln.strip().startswith("traffic_bytes_per_launch:"):
                try:
                    traffic = float(ln.split(":", 1)[1].split()[0])
                    traffic_src = f"{prof} (ncu dram__bytes_read.sum + dram__bytes_write.sum, not measured in this run)"
                except ValueError:
                    pass
    if V == 128:
        kdesc = ("k_reflect_mma (hour-block product on the tensor cores: tcgen05.mma kind::f16 M128 N256, "
                 "128-voxel groups x 256 hours, union rows of the fp16 slab staged by cp.async into 128B-swizzled "
                 "shared memory, split fp16 weights, FP32 accumulation in TMEM, + own term and accumulation)")
    elif V >= 64:
        kdesc = (f"k_reflect_tile<{B // 32}> (hour-block sparse x dense product: union rows of {V}-voxel groups "
                 f"staged in shared memory by cp.async.bulk, merged 4-voxel entries, + accumulation)")
    elif V >= 1:
        kdesc = f"k_reflect_group<{B // 32},{V}> (hour-block sparse x dense product over weighted lists + accumulation)"
    else:
        kdesc = f"k_reflect_block<{B // 32},{args.format}> (hour-block sparse x dense product + accumulation)"
    roof = {"bound": "hbm", "kernel": kdesc,
            "achieved": round(achieved, 2), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 5), "peak_source": peak_src,
            "traffic": traffic, "traffic_source": traffic_src,
            "alg_bytes_per_launch": alg, "launch_ms": round(per_launch_ms, 4),
            "share_of_step": round(refl_ms / max(1e-9, sum(v[0] for v in ktimes.values())), 4),
            "dominant_group": dom[0],
            "gathered_slab_bytes_per_launch": gathered,
            "gather_gbs": round(gathered / (per_launch_ms / 1e3) / 1e9, 1) if per_launch_ms > 0 else None}
    if V >= 1:
        # the product's arithmetic: one FMA per nonzero weight and hour, against
        # the FP32 pipe (148 SMs x 128 FMA/clk x 2 flops at the median SM clock)
        wents = ctx.weighted_entries()
        sm_mhz = clocks.get("sm_mhz") or 0.0
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        fp32_peak = sms * 128 * 2 * sm_mhz * 1e6 / 1e12
        flops = 2.0 * wents * B
        roof["fp32"] = {"useful_flop_per_launch": flops,
                        "achieved_tflops": round(flops / (per_launch_ms / 1e3) / 1e12, 2) if per_launch_ms > 0 else None,
                        "peak_tflops": round(fp32_peak, 1) if fp32_peak else None,
                        "frac": round(flops / (per_launch_ms / 1e3) / 1e12 / fp32_peak, 4)
                        if fp32_peak and per_launch_ms > 0 else None,
                        "peak_note": "FP32 FMA pipe: SMs x 128 lanes x 2 flop x median SM clock under load"}
    if V == 128:
        # executed tensor-core work: two fp16 MMAs (weights hi and lo) of
        # 128 voxels x 256 hours per staged union row
        sm_mhz = clocks.get("sm_mhz") or 0.0
        tens_peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops", 1400.0)))
        tens_src = ("measured" if "bf16_tflops_sustained" in peaks or "bf16_tflops" in peaks
                    else "fallback (sustained under the power cap)")
        dense = 2.0 * 128 * B * float(staged) * 2
        roof["tensor"] = {"executed_flop_per_launch": dense,
                          "achieved_tflops": round(dense / (per_launch_ms / 1e3) / 1e12, 1) if per_launch_ms > 0 else None,
                          "peak_tflops": tens_peak, "peak_source": tens_src,
                          "frac": round(dense / (per_launch_ms / 1e3) / 1e12 / tens_peak, 4) if per_launch_ms > 0 else None,
                          "note": "dense fp16 MMA work including the zero weights of each group's union; the "
                                  "useful work is the fp32 figure (one FMA per nonzero weight and hour)"}
    if 64 <= V < 128:
        # the tile kernel's binding resource: shared-memory reads (one row of
        # B floats + the 18-byte entry per merged entry) against the SM data
        # path, 128 B per clock per SM at the median SM clock of the run
        roof["staged_slab_bytes_per_launch"] = float(staged) * B * 4
        smem_bytes = float(entries) * (B * 4 + 18)
        sm_mhz = clocks.get("sm_mhz") or 0.0
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        smem_peak = sms * 128 * sm_mhz * 1e6 / 1e9
        roof["smem"] = {"bytes_per_launch": smem_bytes,
                        "achieved_gbs": round(smem_bytes / (per_launch_ms / 1e3) / 1e9, 1) if per_launch_ms > 0 else None,
                        "peak_gbs": round(smem_peak, 1) if smem_peak else None,
                        "frac": round(smem_bytes / (per_launch_ms / 1e3) / 1e9 / smem_peak, 4)
                        if smem_peak and per_launch_ms > 0 else None,
                        "peak_note": "148 SMs x 128 B/clk x median SM clock under load"}

    # The binding roof is the one the kernel comes closest to; the top-level
    # figures describe it, and "hbm" keeps the byte roofline either way.
    roof["hbm"] = {"achieved_gbs": roof["achieved"], "peak_gbs": hbm_peak, "frac": roof["frac"],
                   "peak_source": peak_src}
    cands = {"hbm": roof["frac"]}
    for key in ("fp32", "smem", "tensor"):
        if key in roof and roof[key].get("frac") is not None:
            cands[key] = roof[key]["frac"]
    bound = max(cands, key=cands.get)
    if bound == "fp32":
        roof.update({"bound": "fp32", "achieved": roof["fp32"]["achieved_tflops"],
                     "peak": roof["fp32"]["peak_tflops"], "unit": "TFLOP/s", "frac": roof["fp32"]["frac"],
                     "peak_source": "FP32 FMA pipe at the median SM clock (the kernel does not use tensor cores)"})
    elif bound == "tensor":
        roof.update({"bound": "tensor", "achieved": roof["tensor"]["achieved_tflops"],
                     "peak": roof["tensor"]["peak_tflops"], "unit": "TFLOP/s", "frac": roof["tensor"]["frac"],
                     "peak_source": roof["tensor"]["peak_source"]})
    elif bound == "smem":
        roof.update({"bound": "smem", "achieved": roof["smem"]["achieved_gbs"], "peak": roof["smem"]["peak_gbs"],
                     "unit": "GB/s", "frac": roof["smem"]["frac"],
                     "peak_source": "shared-memory data path, 128 B/clk/SM at the median SM clock"})

    # ---- end to end through the host API (pinned host buffers in and out)
    e2e = None
    if True:
        hs = inputs.Scene(scene.name, pinned_copy(scene.grid), scene.width, scene.height, N, T,
                          pinned_copy(scene.pixel_parent), pinned_copy(scene.wall_z), scene.max_height,
                          pinned_copy(scene.sun), pinned_copy(scene.direct), pinned_copy(scene.diffuse),
                          pinned_copy(scene.slopes), pinned_copy(scene.aspects))
        hout = pinned_copy(np.zeros(N, np.float32))
        eopts = dict(neighbor_format=args.format, hour_block=B, accumulation=args.accumulation,
                     group_size=args.group_size, use_graph=1)
        ctx.run_host(hs, hout, **eopts)
        barrier(pg)
        wall = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            ctx.run_host(hs, hout, **eopts)
            wall.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(pg, sum(wall), dev)
        h2d = 4 * (T + N + (N - T) + 2 * N) + 4 * 8760 * 4
        e2e = {"value": world * units * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": 4 * N, "api": "solar_gpu_run_host (C ABI, host buffers)"}

    extra = {}
    if rank == 0 and not args.no_plain:
        # plain per-hour path on the same GPU (the metric's comparison)
        popts = dict(neighbor_format=args.format, hour_block=1, accumulation=2, use_graph=0, time_kernels=0)
        ctx.run_device(scene, d, out, stream=stream.cuda_stream, **popts)   # untimed warm-up run
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        flush.zero_()
        e0.record(stream)
        ctx.run_device(scene, d, out, stream=stream.cuda_stream, **popts)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        plain_ms = e0.elapsed_time(e1)
        extra["plain_per_hour"] = {"ms_per_step": round(plain_ms, 2), "value": units / (plain_ms / 1e3),
                                   "speedup": round(plain_ms / ms_per_step, 2),
                                   "config": "hour_block 1 (one solar + one reflection launch per daylight hour), "
                                             "plain fp32; one untimed warm-up run, then one timed run"}
        ctx.run_device(scene, d, out, stream=stream.cuda_stream, **opts)
        torch.cuda.synchronize(dev)
    if rank == 0:
        # the other neighbor-list format on the same workload (both paths run here)
        ctx.release()
        ofmt = 1 - args.format
        oopts = dict(opts, neighbor_format=ofmt, time_kernels=0)
        ctx.run_device(scene, d, out, stream=stream.cuda_stream, **oopts)
        oms = []
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.run_device(scene, d, out, stream=stream.cuda_stream, **oopts)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            oms.append(e0.elapsed_time(e1))
        extra[f"{FMT_NAMES[ofmt].replace('-', '').lower()}_path"] = {
            "ms_per_step": round(sum(oms) / len(oms), 2), "value": units / (sum(oms) / len(oms) / 1e3),
            "neighbor_format": FMT_NAMES[ofmt]}
        # The annual-sum form of the same path: Stage 1 as above, then each
        # voxel's own hours summed once (FP64) and one sparse product with the
        # sums of its neighbor cells (sum_h sum_g w I = sum_g w sum_h I, the
        # reference's per-hour reflection being linear in I).  Reported beside
        # the headline, whose hour-block product is the method the metric names.
        aopts = dict(opts, reflection=1, time_kernels=0)
        ctx.run_device(scene, d, out, stream=stream.cuda_stream, **aopts)
        ams = []
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.run_device(scene, d, out, stream=stream.cuda_stream, **aopts)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ams.append(e0.elapsed_time(e1))
        extra["annual_sum_path"] = {
            "ms_per_step": round(sum(ams) / len(ams), 2), "value": units / (sum(ams) / len(ams) / 1e3),
            "method": "reflection=annual: Stage 1, then FP64 sums of every voxel's own hours and one sparse "
                      "product over the weighted lists (k_solar_sum, k_reflect_annual)"}
        ctx.run_device(scene, d, out, stream=stream.cuda_stream, **opts)
        torch.cuda.synchronize(dev)
    if rank == 0 and not args.no_check:
        from oracle import oracle as O
        ctx.run_device(scene, d, out, stream=stream.cuda_stream, **opts)
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy().astype(np.float64)
        ranges, psmp = sample_ranges(scene, seed=1)
        orc = O.sample_reference(scene, psmp)
        r = ctx.trace(scene, d, neighbor_format=2)   # both list formats

        def rows(a, b):
            return {"csr_off": r["csr_off"][a:b + 1] - r["csr_off"][a],
                    "csr_ids": r["csr_ids"][r["csr_off"][a]:r["csr_off"][b]],
                    "barle_off": r["barle_off"][a:b + 1] - r["barle_off"][a],
                    "barle": r["barle"][r["barle_off"][a]:r["barle_off"][b]],
                    "shadow": r["shadow"][a:b]}

        extra["list_parity"] = list_parity(O, orc, gpu_sample_lists(ranges, rows), r["shadow"][orc["cells"]], psmp)
        rel = np.abs(got[psmp] - orc["annual"]) / np.maximum(np.abs(orc["annual"]), 1.0)
        extra["error_vs_fp64_oracle_lists"] = {
            "max_rel": float(rel.max()), "mean_rel": float(rel.mean()), "voxels": int(psmp.size),
            "oracle": "FP64 annual-sum oracle on oracle-built lists and shadow words (the sample's own traces and "
                      "traces of every top cell its lists name); denominator floor 1 Wh/m^2"}
        if "annual_sum_path" in extra:
            ctx.run_device(scene, d, out, stream=stream.cuda_stream, **dict(opts, reflection=1, time_kernels=0))
            torch.cuda.synchronize(dev)
            ga = out.cpu().numpy().astype(np.float64)
            rel_a = np.abs(ga[psmp] - orc["annual"]) / np.maximum(np.abs(orc["annual"]), 1.0)
            extra["annual_sum_path"]["error_vs_fp64_oracle_lists"] = {
                "max_rel": float(rel_a.max()), "mean_rel": float(rel_a.mean()), "voxels": int(psmp.size)}
        tot, _ = O.annual_fp64(scene, r["shadow"], r["csr_off"], r["csr_ids"])
        rel = np.abs(got - tot) / np.maximum(np.abs(tot), 1.0)
        extra["error_vs_fp64"] = {"max_rel": float(rel.max()), "mean_rel": float(rel.mean()),
                                  "oracle": "FP64 annual-sum form over every voxel, on the GPU-built neighbor lists "
                                            "and shadow bits (those are checked by list_parity on the sample)"}
        extra["lists_vs_reference"] = lists_vs_reference(O, scene, r)
        del r
    if rank == 0:
        # caller-side voxelization of the heightmap: the reference's host
        # restatement (numpy) against solar_gpu_voxelize, same arrays
        heights = scene.grid.reshape(scene.height, scene.width)
        t0 = time.perf_counter()
        inputs.voxelize(heights, 1.0)
        host_s = time.perf_counter() - t0
        g = torch.from_numpy(scene.grid).to(dev)
        ctx.voxelize(g, scene.width, scene.height, 1.0)   # warm (buffers)
        torch.cuda.synchronize(dev)
        gms = []
        for _ in range(3):
            t0 = time.perf_counter()
            v = ctx.voxelize(g, scene.width, scene.height, 1.0)
            torch.cuda.synchronize(dev)
            gms.append((time.perf_counter() - t0) * 1e3)
        same = bool(torch.equal(v["pixel_parent"].cpu(), torch.from_numpy(scene.pixel_parent)))
        extra["voxelize"] = {"gpu_ms": round(sorted(gms)[1], 3), "host_numpy_ms": round(host_s * 1e3, 1),
                             "voxels": v["num_total"], "pixel_parent_equal": same,
                             "how": "solar_gpu_voxelize (count, scan, write; wall clock around the synchronous "
                                    "call, median of 3) against the numpy restatement of src/voxelization.cpp"}
        del g, v
    cpu = None
    steps_per_ray = nst = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        rng = np.random.default_rng(0)
        ns = min(N, 20000)
        smp = np.sort(rng.choice(N, ns, replace=False))
        r = O.cpu_sample(scene, smp, hblock=128)
        cpu = {"value": r["voxel_hours_per_s"], "unit": UNIT, "cores": r["threads"], "kind": "port",
               "sample": (f"FP64 oracle, per-hour method: full trace of {ns} random voxels ({r['trace_s']:.2f} s), "
                          f"top-cell solar table for one {r['hblock']}-hour block ({r['table_s']:.2f} s), "
                          f"per-hour reflection sums of the {ns} voxels for that block ({r['sums_s']:.2f} s); "
                          f"scaled to {N} voxels x {r['hours']} h")}
        # the workload's mean DDA steps per ray, counted by the oracle on a sample
        nst = min(ns, 2000)
        steps_per_ray = float(O.trace_steps(scene, smp[:nst]).astype(np.float64).mean())

    if rank == 0 and world == 1 and not (args.no_config3 and args.no_config4):
        del d, out
        ctx.release()
        if not args.no_config4:
            extra["config4"] = run_config4(args)
        if not args.no_config3:
            extra["config3"] = run_config3(args, ctx, dev, stream, flush)
        ctx.release()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_desc(scene, args.workload), "voxels": N, "daylight_hours": Hd,
                       "neighbor_format": FMT_NAMES[args.format], "hour_block": B,
                       "accumulation": ACC_NAMES[args.accumulation],
                       "l2": "256 MiB buffer written between timed steps (outside the events)",
                       "parallelism": f"{world} independent replica(s), no exchange"},
            "e2e": e2e, "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
            "stage_ms": {g: round(v[0] / args.steps, 3) for g, v in ktimes.items()},
        }
        if "trace" in ktimes:
            # Stage 1 in its own units: rays = voxels x 2592 directions per run
            t_trace = ktimes["trace"][0] / args.steps / 1e3
            rays = float(N) * N_DIRS
            st1 = {"rays_per_run": rays, "rays_per_s": rays / t_trace, "trace_ms": round(t_trace * 1e3, 3)}
            if steps_per_ray is not None:
                st1.update({"dda_steps_per_ray": round(steps_per_ray, 3),
                            "dda_steps_per_s": steps_per_ray * rays / t_trace,
                            "steps_source": f"mean DDA steps per ray of the reference's loop, counted by the oracle "
                                            f"on {nst} random voxels (upper rays above their cone's bound end "
                                            f"early here, so fewer steps run)"})
            line["stage1"] = st1
        line.update(extra)
        print(json.dumps(line), flush=True)
    ctx.close()


# ---------------------------------------------------------------- reference arm

class quiet_stdout:
    """Sends file descriptor 1 to /dev/null (the reference prints progress from C++)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        try:   # C stdio may still hold what was printed: let it go to /dev/null too
            import ctypes
            ctypes.CDLL(None).fflush(None)
        except OSError:
            pass
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def run_reference(args, world, rank, local, pg):
    if rank != 0:
        return
    from oracle import oracle as O
    from solargpu_b200 import inputs
    if O.ref_gpu() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsolarref.so was not built"}))
        return
    # One full annual run of the workload per step (24 s for the 1024 x 1024
    # city through the uncompressed entry point); a smaller workload of the
    # same generator can be named with --ref-workload.
    ref_workload = args.ref_workload or args.workload
    scene = inputs.make_scene(ref_workload)
    comp = args.format == 1
    Hd = int(((scene.sun[:, 1] - np.float32(1e-8)) >= 1.0).sum())
    units = float(scene.num_total) * Hd
    for _ in range(args.warmup):
        with quiet_stdout():
            O.ref_irradiance(scene, comp)
    wall = []
    for _ in range(args.steps):
        with quiet_stdout():
            t0 = time.perf_counter()
            O.ref_irradiance(scene, comp)   # synchronous stock API (H2D, both stages, D2H)
            wall.append(time.perf_counter() - t0)
    sec = sum(wall)
    value = units * args.steps / sec
    N, T = scene.num_total, scene.num_top
    # grid, slopes, aspects, pixel_parent, wall_z; sun (az, alt), dense sun bin,
    # DNI, DHI per hour of the year (device_globals.cu:45-48) and the Perez table
    h2d = 4 * (T + 3 * N + (N - T)) + 8760 * (8 + 4 + 4 + 4) + 6 * 8 * 4
    d2h = 4 * N
    desc = ("reference CUDA pipeline (src/cuda/*.cu, sm_100a build of the unmodified sources) through its stock "
            f"API solar_gpu::{'compressed' if comp else 'uncompressed'}_gpu_irradiance, host buffers in/out; "
            f"one full annual run of {ref_workload} per step"
            + (f" (bounded sample of {args.workload})" if ref_workload != args.workload else ""))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload_desc(scene, ref_workload), "voxels": scene.num_total,
                       "daylight_hours": Hd, "neighbor_format": FMT_NAMES[args.format],
                       "warmup_runs": args.warmup},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": desc + " (the reference has no CPU path; its host thread drives the GPU)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "note": "the stock API copies inside every call: the caller's arrays and the 8760-hour "
                            "tables in, the raster out (counted here); Stage 1 also stages its raw hit rows to "
                            "the host and uploads the assembled lists (not counted)"}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, local, pg)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
