"""Multi-tile runner and autotuner: CPU checks of the tile set and the tuner
logic, and a GPU check that the threaded multi-tile pass reproduces
single-tile runs."""
import dataclasses
import json

import numpy as np
import pytest

from solargpu_b200 import inputs, tiles


def test_tile_set_is_seeded_and_in_range():
    a = tiles.tile_configs(32, seed=3)
    b = tiles.tile_configs(32, seed=3)
    assert a == b
    assert tiles.tile_configs(32, seed=4) != a
    for c in a:
        assert 128 <= c.size <= 1024 and c.size % 16 == 0
        assert 35.0 <= c.lat <= 60.0 and -10.0 <= c.lon <= 30.0
        assert c.tz == int(round(c.lon / 15.0))
        assert c.n_buildings >= 1 and c.n_trees >= 1
    sizes = [c.size for c in a]
    assert min(sizes) < 256 and max(sizes) > 512      # spans the range


def test_autotuner_picks_fastest_once_per_bucket(tmp_path):
    cands = [dict(hour_block=b) for b in (64, 128, 256)]
    cost = {64: 3.0, 128: 1.0, 256: 2.0}
    calls = []

    def measure(c):
        calls.append(c["hour_block"])
        return cost[c["hour_block"]]

    path = str(tmp_path / "tune.json")
    t = tiles.Autotuner(cands, path=path)
    assert t.choose(20, measure) == {"hour_block": 128}
    assert t.choose(20, measure) == {"hour_block": 128}
    assert calls == [64, 128, 256]                    # measured once
    assert json.load(open(path)) == {"20": {"hour_block": 128}}
    t2 = tiles.Autotuner(cands, path=path)            # reloaded table: no trials
    assert t2.choose(20, lambda c: pytest.fail("measured again")) == {"hour_block": 128}


@pytest.mark.gpu
def test_multi_tile_pass_matches_single_runs():
    import torch
    from solargpu_b200 import api
    cfgs = [inputs.DsmConfig(f"t{i}", n, 2, 8, lat=40.0 + 5 * i, lon=5.0 * i, tz=0, seed=70 + i)
            for i, n in enumerate((64, 80, 96))]
    scenes = [inputs.make_scene(c) for c in cfgs]
    r = tiles.run_tiles(scenes, params=tiles.DEFAULT, workers=2, keep_outputs=True)
    with api.Context(0) as ctx:
        for s, t in zip(scenes, r["tiles"]):
            d = tiles._device_arrays(s, torch.device("cuda", 0))
            out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
            ctx.run_device(s, d, out, accumulation=1, **tiles.DEFAULT)
            torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy(), t["out"]), s.name
    assert r["voxel_hours"] > 0 and r["wall_s"] > 0
    tuned = tiles.run_tiles(scenes, tuner=tiles.Autotuner(), workers=1, keep_outputs=True)
    for a, b in zip(r["tiles"], tuned["tiles"]):
        rel = np.abs(a["out"].astype(np.float64) - b["out"]) / np.maximum(np.abs(a["out"]), 1.0)
        assert rel.max() <= 1e-5
        assert b["params"] in [dict(c) for c in tiles.CANDIDATES]


@pytest.mark.gpu
def test_batch_equals_tile_by_tile(cuda_lib):
    """Four uneven tiles (own sites and hourly series) through one batch --
    every hour loop a branch of one CUDA graph -- give the same rasters, bit
    for bit, as running each tile alone with the same options, and stay within
    1e-4 of the FP64 oracle."""
    import torch
    from oracle import oracle as O
    from solargpu_b200 import api, inputs, tiles
    cfgs = tiles.tile_configs(4, seed=3)
    scenes = [inputs.make_scene(dataclasses.replace(c, size=min(c.size, 160), n_buildings=min(c.n_buildings, 20),
                                                    n_trees=min(c.n_trees, 60)))
              for c in cfgs]
    r = tiles.run_tiles_batched(scenes, runs=1, keep_outputs=True)
    for s, got in zip(scenes, r["outs"]):
        out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
        with api.Context(0) as ctx:
            ctx.run_device(s, tiles._device_arrays(s, torch.device("cuda:0")), out, accumulation=1,
                           **tiles.DEFAULT)
        torch.cuda.synchronize()
        assert np.array_equal(got, out.cpu().numpy()), s.name
        bins = O.sky_bins(s.sun)
        off, ids, sh = O.trace(s, bins)
        want, _ = O.annual_fp64(s, sh, off, ids)
        assert (np.abs(got.astype(np.float64) - want) / np.maximum(want, 1.0)).max() <= 1e-4, s.name
