"""CPU checks of the oracle and of the caller-side inputs against the
reference's own code (golden fixtures made by tests/golden/make_golden.py)."""
import hashlib
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, load_scene, oracle_trace


def _lists(d, off_key="off", ids_key="ids"):
    off, ids = d[off_key], d[ids_key]
    return [ids[off[i]:off[i + 1]] for i in range(off.size - 1)]


def test_barle_encoder_matches_reference(oracle_lib):
    """Byte-exact to src/barle_compression.cpp:156-187 on lists covering every
    width class, runs longer than 255, the absorb rule, and empty lists."""
    d = np.load(os.path.join(GOLDEN, "barle_golden.npz"))
    lists = _lists(d)
    ref = [d["bytes"][d["boff"][i]:d["boff"][i + 1]].tobytes() for i in range(len(lists))]
    for ids, want in zip(lists, ref):
        assert oracle_lib.barle_encode(ids) == want


def test_barle_roundtrip(oracle_lib):
    d = np.load(os.path.join(GOLDEN, "barle_golden.npz"))
    for ids in _lists(d):
        dec = oracle_lib.barle_decode(oracle_lib.barle_encode(ids))
        want = np.unique(ids.astype(np.uint32))[::-1]
        assert np.array_equal(dec, want)


def test_barle_csr_encoder_concatenates(oracle_lib):
    d = np.load(os.path.join(GOLDEN, "barle_golden.npz"))
    boff, buf = oracle_lib.barle_encode_csr(d["off"], d["ids"])
    assert np.array_equal(boff, d["boff"])
    assert np.array_equal(buf, d["bytes"])


@pytest.mark.parametrize("cut", [1, 2, 3, 4])
def test_barle_decoder_rejects_truncated(oracle_lib, cut):
    enc = oracle_lib.barle_encode(np.arange(1, 300, 7, dtype=np.int32))
    with pytest.raises(ValueError):
        oracle_lib.barle_decode(enc[:-cut] if cut < 4 else enc[:2])


def test_barle_decoder_rejects_bad_code(oracle_lib):
    enc = bytearray(oracle_lib.barle_encode(np.array([5, 3, 1], np.int32)))
    enc[0] = (enc[0] & 0x1F) | (5 << 5)   # first 3-bit code -> 5 (unused)
    with pytest.raises(ValueError):
        oracle_lib.barle_decode(bytes(enc))


@pytest.mark.parametrize("name", ["dsm64", "dsm160"])
def test_sky_bins_match_reference(oracle_lib, name):
    s = load_scene(name)
    g = np.load(os.path.join(GOLDEN, f"sky_{name}.npz"))
    b = oracle_lib.sky_bins(s.sun)
    assert np.array_equal(b["full_to_dense"], g["full_to_dense"])
    assert np.array_equal(b["sun_dense_idx"], g["sun_dense_idx"])
    assert np.array_equal(b["nudged"], g["nudged"])
    assert [b["hsize"], b["vsize"], b["vsize_full"], b["active"], b["words8"]] == list(g["meta"])


def test_sun_positions_match_reference():
    from solargpu_b200 import inputs
    g = np.load(os.path.join(GOLDEN, "sky_dsm64.npz"))
    c = inputs.CONFIGS["dsm64"]
    assert np.array_equal(inputs.sun_positions(c.lon, c.lat, c.tz), g["ref_sun"][:8760])


@pytest.mark.parametrize("name", ["dsm64", "dsm160"])
def test_voxelization_matches_reference(name):
    """The caller-side voxelization agrees with src/voxelization.cpp:10-97
    (parents and heights exactly; angles to float rounding)."""
    from solargpu_b200 import inputs
    s = load_scene(name)
    g = np.load(os.path.join(GOLDEN, f"voxel_{name}.npz"))
    par, z, asp = inputs.detect_wall_voxels(s.grid.reshape(s.height, s.width))
    assert np.array_equal(par, g["parent"])
    assert np.array_equal(z, g["z"])
    assert np.allclose(asp, g["aspect"], rtol=0, atol=2e-6)
    sl, ta = inputs.top_slope_aspect(s.grid.reshape(s.height, s.width))
    assert np.allclose(sl, g["slope"], rtol=0, atol=2e-6)
    assert np.allclose(ta, g["top_aspect"], rtol=0, atol=2e-6)


def test_scene_generator_is_deterministic():
    from solargpu_b200 import inputs
    a = inputs.make_scene("dsm64")
    b = load_scene("dsm64")
    for k, v in a.arrays().items():
        assert np.array_equal(v, b.arrays()[k]), k


def test_trace_lists_are_first_occurrence_unique(scene64):
    bins, off, ids, sh = oracle_trace(scene64)
    assert off[0] == 0 and off[-1] == ids.size
    assert ids.min() >= 1 and ids.max() <= scene64.num_top
    for v in range(0, scene64.num_total, 97):
        l = ids[off[v]:off[v + 1]]
        assert np.unique(l).size == l.size
    assert sh.shape == (scene64.num_total, (bins["active"] + 31) // 32)


@pytest.mark.parametrize("name", ["dsm64", "dsm160"])
def test_oracle_trace_matches_reference_gpu_golden(name):
    """Oracle DDA vs the reference CUDA kernel's own output (digests of the
    full CSR ids, ba-RLE stream and shadow bitmap, made on a B200)."""
    path = os.path.join(GOLDEN, f"ref_stage1_{name}.npz")
    if not os.path.exists(path):
        pytest.skip("reference GPU fixture not generated yet")
    from oracle import oracle as O
    g = np.load(path)
    s = load_scene(name)
    bins, off, ids, sh = oracle_trace(s)
    assert np.array_equal(np.diff(off).astype(np.int32), g["counts"])
    assert hashlib.sha256(ids.astype(np.int32).tobytes()).hexdigest() == str(g["sha_ids"])
    boff, buf = O.barle_encode_csr(off, ids)
    assert hashlib.sha256(buf.tobytes()).hexdigest() == str(g["sha_barle"])
    svf8 = np.zeros((int(g["svf_words8"]), s.num_total), np.uint8)
    bytes_ = sh.view(np.uint8).reshape(s.num_total, -1)[:, :int(g["svf_words8"])]
    svf8[:] = bytes_.T
    assert hashlib.sha256(svf8.tobytes()).hexdigest() == str(g["sha_svf"])


def test_oracle_trace_matches_reference_gpu_blocks_dsm1024():
    """Oracle DDA on the 1024 x 1024 city against the reference CUDA viewshed
    stage's own output (per-block digests made on a B200): three seeded blocks
    of 4096 voxels (one of them the last, wall voxels), list lengths, CSR ids,
    ba-RLE sizes and bytes and the shadow bitmap."""
    path = os.path.join(GOLDEN, "ref_stage1_blocks_dsm1024.npz")
    if not os.path.exists(path):
        pytest.skip("reference GPU fixture not generated yet")
    sys.path.insert(0, GOLDEN)
    import make_golden as MG
    from oracle import oracle as O
    from solargpu_b200 import inputs
    g = np.load(path)
    s = inputs.make_scene("dsm1024")
    assert MG.scene_digest(s) == str(g["scene"]), "the generator no longer makes the fixture's scene"
    n, B = int(g["num_total"]), int(g["block"])
    assert n == s.num_total
    nb = (n + B - 1) // B
    rng = np.random.default_rng(11)
    bins = O.sky_bins(s.sun)
    for b in sorted(set(rng.choice(nb - 1, 2, replace=False).tolist() + [nb - 1])):
        v0, v1 = b * B, min(n, (b + 1) * B)
        off, ids, sh = O.trace(s, bins, v0, v1)
        boff, buf = O.barle_encode_csr(off, ids)
        w8 = int(g["svf_words8"])
        svf8 = np.ascontiguousarray(sh.view(np.uint8).reshape(v1 - v0, -1)[:, :w8].T)
        got = MG.block_digests(off, ids, boff, buf, svf8, 0, v1 - v0)
        assert got == [str(x) for x in g["digests"][b]], (b, v0, v1)


def test_fp64_forms_agree(scene64):
    """Annual-sum form and per-hour form of the FP64 oracle (linearity)."""
    from oracle import oracle as O
    bins, off, ids, sh = oracle_trace(scene64)
    tot, dd = O.annual_fp64(scene64, sh, off, ids)
    v0, v1 = 100, 400
    hr = O.hourly_fp64(scene64, sh, off, ids, v0, v1, hblock=97)
    assert np.allclose(hr, tot[v0:v1], rtol=1e-12, atol=0)
    v0, v1 = scene64.num_top + 10, scene64.num_top + 200
    hr = O.hourly_fp64(scene64, sh, off, ids, v0, v1, hblock=64)
    assert np.allclose(hr, tot[v0:v1], rtol=1e-12, atol=0)


@pytest.mark.parametrize("name", ["dsm64", "dsm160"])
def test_fp64_oracle_matches_reference_annual_output(name):
    """The FP64 irradiance oracle against the reference pipeline's own annual
    rasters (both instances, run on a B200 through the stock API): they agree
    to the reference's FP32 per-hour accumulation error, far inside 1e-4."""
    path = os.path.join(GOLDEN, f"ref_annual_{name}.npz")
    if not os.path.exists(path):
        pytest.skip("reference GPU fixture not generated yet")
    from oracle import oracle as O
    g = np.load(path)
    s = load_scene(name)
    bins, off, ids, sh = oracle_trace(s)
    tot, _ = O.annual_fp64(s, sh, off, ids)
    for key in ("uncompressed", "compressed"):
        rel = np.abs(g[key].astype(np.float64) - tot) / tot
        assert rel.max() < 2e-5, (key, rel.max())
        assert rel.mean() < 2e-6, (key, rel.mean())


def test_lists_cache_roundtrip_and_fingerprints(tmp_path):
    """The on-disk Stage 1 cache keeps the lists exactly and refuses scenes
    whose geometry or sun positions differ from the traced one."""
    import dataclasses
    from solargpu_b200 import cache
    s = load_scene("dsm64")
    bins, off, ids, sh = oracle_trace(s)
    r = {"csr_off": off.astype(np.int64), "csr_ids": ids.astype(np.int32), "shadow": sh,
         "shadow_words": sh.shape[1], "active_bins": bins["active"]}
    p = str(tmp_path / "t.npz")
    cache.save_lists(p, r, s)
    got = cache.load_lists(p, s)
    assert np.array_equal(got["csr_off"], r["csr_off"]) and np.array_equal(got["csr_ids"], r["csr_ids"])
    assert np.array_equal(got["shadow"], sh) and got["active_bins"] == bins["active"]
    # new hourly irradiance: same fingerprints
    s2 = dataclasses.replace(s, direct=s.direct * np.float32(0.5))
    cache.load_lists(p, s2)
    s3 = dataclasses.replace(s, grid=s.grid + np.float32(1.0))
    with pytest.raises(ValueError):
        cache.load_lists(p, s3)
    sun = s.sun.copy()
    sun[100:200, 0] += np.float32(1.0)
    with pytest.raises(ValueError):
        cache.load_lists(p, dataclasses.replace(s, sun=sun))
    from oracle import oracle as O
    boff, bbytes = O.barle_encode_csr(off, ids)
    rb = {"barle_off": boff, "barle": bbytes, "shadow": sh, "shadow_words": sh.shape[1], "active_bins": bins["active"]}
    cache.save_lists(p, rb, s)
    gb = cache.load_lists(p)
    assert np.array_equal(gb["barle"], bbytes) and "csr_off" not in gb


# ---- DDA known answers on hand-made heightmaps (viewshed_kernels.cu:7-59) --------------------
# Answers worked out by hand from the ray geometry: origin = cell corner + 2 * Cdir, the start
# cell is never tested, a hit is height - z_ray > 0.01 at the cell entered, an upward ray stops
# above the maximum height, a downward one below 0, and a tie tMaxX == tMaxY steps y.

def _dir(az_deg: float, el_deg: float):
    """(cx, cy, cz) for azimuth/elevation in the reference's convention: x = cos e sin az,
    y = -cos e cos az, z = sin e."""
    a, e = np.radians(az_deg), np.radians(el_deg)
    return (np.float32(np.cos(e) * np.sin(a)), np.float32(-np.cos(e) * np.cos(a)), np.float32(np.sin(e)))


def _grid(towers=()):
    g = np.zeros((16, 16), np.float32)
    for x, y, h in towers:
        g[y, x] = h
    return g


def test_dda_flat_plane_has_no_hits():
    from oracle import oracle as O
    g = _grid()
    for az in np.arange(2.5, 360.0, 5.0):
        for el in np.arange(-87.5, 90.0, 5.0):
            for gx, gy in ((0, 0), (7, 9), (15, 15)):
                assert O.trace_one(g, 0.0, gx, gy, 0.0, _dir(az, el), el > 0) == 0


def test_dda_single_tower():
    from oracle import oracle as O
    g = _grid([(10, 5, 10.0)])
    east = lambda el: (np.float32(np.cos(np.radians(el))), np.float32(0.0), np.float32(np.sin(np.radians(el))))
    # at 60 degrees the ray is 8.66 m high entering x = 10: hit (id 10 + 5 * 16 + 1)
    assert O.trace_one(g, 10.0, 5, 5, 0.0, east(60.0), True) == 91
    # at 70 degrees it passes 10 m (the maximum height) over x = 9 and stops
    assert O.trace_one(g, 10.0, 5, 5, 0.0, east(70.0), True) == 0
    # westward there is nothing to hit before the grid edge
    west = (np.float32(-np.cos(np.radians(10.0))), np.float32(0.0), np.float32(np.sin(np.radians(10.0))))
    assert O.trace_one(g, 10.0, 5, 5, 0.0, west, True) == 0
    # from the tower top downward to the west: the ray goes below 0 before anything is higher
    down = (np.float32(-np.cos(np.radians(30.0))), np.float32(0.0), np.float32(-0.5))
    assert O.trace_one(g, 10.0, 10, 5, 10.0, down, False) == 0


def test_dda_start_cell_is_not_tested():
    from oracle import oracle as O
    c = (np.float32(np.cos(np.radians(10.0))), np.float32(0.0), np.float32(np.sin(np.radians(10.0))))
    # origin x = 5 + 2 cos(10 deg) = 6.97: the start cell is (6, 5); a tower there is skipped
    assert O.trace_one(_grid([(6, 5, 10.0)]), 10.0, 5, 5, 0.0, c, True) == 0
    assert O.trace_one(_grid([(7, 5, 10.0)]), 10.0, 5, 5, 0.0, c, True) == 7 + 5 * 16 + 1


def test_dda_grid_edge():
    from oracle import oracle as O
    # along the last column toward -y: start cell (15, 13), the first cell entered is (15, 12)
    c = (np.float32(0.0), np.float32(-np.cos(np.radians(10.0))), np.float32(np.sin(np.radians(10.0))))
    assert O.trace_one(_grid([(15, 12, 10.0)]), 10.0, 15, 15, 0.0, c, True) == 15 + 12 * 16 + 1
    # from the corner outward: the first step leaves the grid
    out = (np.float32(-0.6), np.float32(-0.6), np.float32(0.5291503))
    assert O.trace_one(_grid([(0, 0, 10.0)]), 10.0, 0, 0, 0.0, out, True) == 0


def test_dda_tie_steps_y_first():
    from oracle import oracle as O
    # cx == cy: from origin (6.41, 6.41) tMaxX == tMaxY exactly, and the tie steps y into (6, 7)
    c = (np.float32(0.7066), np.float32(0.7066), np.float32(0.0349))
    assert O.trace_one(_grid([(6, 7, 10.0)]), 10.0, 5, 5, 0.0, c, True) == 6 + 7 * 16 + 1
    # stepping y first, the ray never enters (7, 6): it goes (6, 7), (7, 7), (7, 8), ...
    assert O.trace_one(_grid([(7, 6, 10.0)]), 10.0, 5, 5, 0.0, c, True) == 0
    assert O.trace_one(_grid([(7, 7, 10.0)]), 10.0, 5, 5, 0.0, c, True) == 7 + 7 * 16 + 1


def test_voxel_dump_format(tmp_path, scene64):
    """The voxel dump of the reference CLI (src/main.cpp:44-67): two int32
    counts, then per voxel float32 x, y, z, irradiance; z is the cell height
    for a top voxel and the wall height for a wall voxel."""
    from solargpu_b200 import outputs
    s = scene64
    irr = np.linspace(1.0, 2.0, s.num_total).astype(np.float32)
    p = str(tmp_path / "v.bin")
    outputs.write_voxel_dump(p, s, irr)
    raw = open(p, "rb").read()
    assert len(raw) == 8 + 16 * s.num_total
    n, t = np.frombuffer(raw[:8], "<i4")
    assert (n, t) == (s.num_total, s.num_top)
    rec = np.frombuffer(raw[8:], "<f4").reshape(-1, 4)
    for i in (0, 1, s.num_top - 1, s.num_top, s.num_total - 1):
        top = int(s.pixel_parent[i])
        gx, gy = top % s.width, top // s.width
        z = s.grid[gy * s.width + gx] if i < s.num_top else s.wall_z[i - s.num_top]
        assert list(rec[i]) == [np.float32(gx), np.float32(gy), np.float32(z), irr[i]]
    n2, t2, r2 = outputs.read_voxel_dump(p)
    assert (n2, t2) == (n, t) and np.array_equal(r2["val"], irr)
    outputs.write_raster(str(tmp_path / "r.npy"), s, irr)
    r = np.load(str(tmp_path / "r.npy"))
    assert r.shape == (s.height, s.width) and np.array_equal(r.ravel(), irr[:s.num_top])
