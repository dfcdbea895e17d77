"""GPU parity: the CUDA library (through its C ABI) against the oracle and,
when it was built, against the reference CUDA pipeline itself.

Integer work (neighbor ids, shadow bits, ba-RLE bytes) must be bit-exact.
Annual irradiance must be within REL_TOL of the FP64 oracle per voxel."""
import numpy as np
import pytest

from conftest import device_arrays, load_scene, oracle_trace

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4          # max relative error per voxel vs the FP64 oracle
FLOOR = 1.0             # Wh/m^2 denominator floor (all annual values here are > 1e5)


@pytest.fixture(scope="module")
def ctx(cuda_lib):
    from solargpu_b200 import api
    c = api.Context(0)
    yield c
    c.close()


def fp64_reference(scene):
    from oracle import oracle as O
    bins, off, ids, sh = oracle_trace(scene)
    tot, _ = O.annual_fp64(scene, sh, off, ids)
    return tot


def rel_err(got, want):
    return np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), FLOOR)


@pytest.mark.parametrize("name", ["dsm64", "dsm160"])
def test_trace_matches_oracle(ctx, name):
    from oracle import oracle as O
    s = load_scene(name)
    bins, off, ids, sh = oracle_trace(s)
    r = ctx.trace(s, device_arrays(s))
    assert r["active_bins"] == bins["active"]
    np.testing.assert_array_equal(r["csr_off"], off)
    np.testing.assert_array_equal(r["csr_ids"], ids)
    np.testing.assert_array_equal(r["shadow"], sh)
    boff, buf = O.barle_encode_csr(off, ids)
    np.testing.assert_array_equal(r["barle_off"], boff)
    np.testing.assert_array_equal(r["barle"], buf)


def test_trace_nonfinite_heights_match_oracle(ctx):
    """Heights of +inf, -inf and NaN, in grid cells (border and interior) and
    in wall voxels.  The tracer stops rays on a +inf border around its copy
    of the heightmap; these inputs must still give the reference's lists and
    shadow bits (viewshed_kernels.cu:31-58: a NaN or +inf start height never
    hits, a -inf one hits the first finite cell, NaN cells are passed over)."""
    import dataclasses
    s = load_scene("dsm64")
    g = s.grid.copy()
    W = s.width
    for x, y, v in [(10, 12, np.inf), (30, 31, -np.inf), (40, 20, np.nan), (0, 0, np.inf), (63, 63, np.nan),
                    (5, 50, -np.inf), (63, 7, np.inf), (22, 0, np.nan)]:
        g[y * W + x] = v
    wz = s.wall_z.copy()
    wz[[0, 7, 19, 101, 333, 777]] = [np.inf, -np.inf, np.nan, np.inf, -np.inf, np.nan]
    s2 = dataclasses.replace(s, name="dsm64_nonfinite", grid=g, wall_z=wz)
    bins, off, ids, sh = oracle_trace(s2)
    r = ctx.trace(s2, device_arrays(s2))
    np.testing.assert_array_equal(r["csr_off"], off)
    np.testing.assert_array_equal(r["csr_ids"], ids)
    np.testing.assert_array_equal(r["shadow"], sh)


@pytest.mark.parametrize("max_height", ["true", "below", "nan"])
def test_trace_early_exit_on_towers_matches_oracle(ctx, max_height):
    """Upper rays end early once they pass the early-exit bound of their cone
    of directions (cone.cu).  A non-square field of low blocks with a few tall
    towers, NaN and +inf cells, traced with the scene maximum as given, with a
    maximum below the tallest tower (the reference's range test then ends rays
    that would still hit it) and with a NaN maximum (the range test never
    fires): lists and shadow bits equal the oracle's."""
    import dataclasses
    from oracle import oracle as O
    from solargpu_b200 import inputs
    rng = np.random.default_rng(7)
    h = (rng.random((83, 117)) * 4.0).astype(np.float32)
    for _ in range(40):
        y, x = rng.integers(0, 80), rng.integers(0, 114)
        h[y:y + rng.integers(1, 4), x:x + rng.integers(1, 4)] += np.float32(rng.random() * 25.0)
    for y, x, v in [(5, 9, 60.0), (70, 100, 45.0), (41, 58, 52.0)]:
        h[y, x] = v
    s = inputs.scene_from_heightmap("towers", h, 1.0, 15.592, 46.543, 1)
    g = s.grid.copy()
    g[20 * 117 + 3], g[60 * 117 + 60] = np.nan, np.inf   # after voxelization, which wants finite heights
    mz = {"true": s.max_height, "below": np.float32(30.0), "nan": np.float32(np.nan)}[max_height]
    s = dataclasses.replace(s, name="towers_" + max_height, grid=g, max_height=mz)
    bins, off, ids, sh = oracle_trace(s)
    r = ctx.trace(s, device_arrays(s), neighbor_format=2)
    np.testing.assert_array_equal(r["csr_off"], off)
    np.testing.assert_array_equal(r["csr_ids"], ids)
    np.testing.assert_array_equal(r["shadow"], sh)
    boff, bbytes = O.barle_encode_csr(off, ids)
    np.testing.assert_array_equal(r["barle_off"], boff)
    np.testing.assert_array_equal(r["barle"], bbytes)


def test_trace_without_early_exit_tables_gives_the_same_lists(ctx, scene160, monkeypatch):
    """SGB_CONE=0 leaves one table whose bound is the scene maximum (the
    reference's range test alone): the lists and shadow bits are the same
    bits as with the cone tables."""
    d = device_arrays(scene160)
    a = ctx.trace(scene160, d, neighbor_format=2)
    monkeypatch.setenv("SGB_CONE", "0")
    b = ctx.trace(scene160, d, neighbor_format=2)
    for k in ("csr_off", "csr_ids", "barle_off", "barle", "shadow"):
        np.testing.assert_array_equal(a[k], b[k])


def test_dedupe_second_pass_gives_the_same_lists(cuda_lib, scene160):
    """The first-occurrence dedupe first runs with small hash sets and hands
    the rows it gives up on to a second pass with large ones.  With the
    first pass's probe bound forced down to one probe (SGB_DEDUPE_PROBES=1)
    most rows take the second pass, after part of them was already compacted:
    the lists must still equal the oracle's.  Runs in a child process so the
    setting stays out of the other tests."""
    import os
    import subprocess
    import sys
    from conftest import ROOT
    code = (
        "import sys, numpy as np; sys.path.insert(0, 'tests'); sys.path.insert(0, '.');"
        "from conftest import load_scene, device_arrays, oracle_trace;"
        "from solargpu_b200 import api;"
        "s = load_scene('dsm160'); bins, off, ids, sh = oracle_trace(s);"
        "c = api.Context(0); r = c.trace(s, device_arrays(s), neighbor_format=0);"
        "assert np.array_equal(r['csr_off'], off) and np.array_equal(r['csr_ids'], ids);"
        "assert np.array_equal(r['shadow'], sh); print('same lists')")
    env = dict(os.environ, SGB_DEDUPE_PROBES="1")
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0 and "same lists" in p.stdout, p.stdout + p.stderr


def test_union_second_pass_gives_the_same_result(cuda_lib, scene160, tmp_path):
    """The group unions of the tensor-core kernel are built by a first pass
    with room for 8192 cells a group and a second pass, with room for 16384,
    for the groups the first hands on.  With every group handed on
    (SGB_UNION_SECOND_PASS=1) the irradiance must be bit-identical to the
    default run.  Runs in a child process so the setting stays out of the
    other tests."""
    import os
    import subprocess
    import sys
    import torch
    from solargpu_b200 import api
    from conftest import ROOT
    out = torch.zeros(scene160.num_total, dtype=torch.float32, device="cuda:0")
    with api.Context(0) as c:
        c.run_device(scene160, device_arrays(scene160), out, neighbor_format=0, hour_block=256, group_size=128)
    want = out.cpu().numpy()
    code = (
        "import sys, numpy as np, torch; sys.path.insert(0, 'tests'); sys.path.insert(0, '.');"
        "from conftest import load_scene, device_arrays;"
        "from solargpu_b200 import api;"
        "s = load_scene('dsm160'); out = torch.zeros(s.num_total, dtype=torch.float32, device='cuda:0');"
        "c = api.Context(0); c.run_device(s, device_arrays(s), out, neighbor_format=0, hour_block=256, group_size=128);"
        "np.save(sys.argv[1], out.cpu().numpy()); print('ran')")
    path = str(tmp_path / "second_pass.npy")
    env = dict(os.environ, SGB_UNION_SECOND_PASS="1")
    p = subprocess.run([sys.executable, "-c", code, path], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0 and "ran" in p.stdout, p.stdout + p.stderr
    got = np.load(path)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))


def test_trace_chunked_equals_single(ctx, scene160):
    dev = device_arrays(scene160)
    a = ctx.trace(scene160, dev)
    b = ctx.trace(scene160, dev, chunk_voxels=3001)
    for k in ("csr_off", "csr_ids", "barle_off", "barle", "shadow"):
        np.testing.assert_array_equal(a[k], b[k])


def test_trace_matches_reference_kernel(ctx, scene64):
    """Bit-exact against the reference's own viewshed stage rebuilt for sm_100a."""
    from oracle import oracle as O
    if O.ref_gpu() is None:
        pytest.skip("reference CUDA pipeline not built")
    ref = O.ref_stage1(scene64)
    r = ctx.trace(scene64, device_arrays(scene64))
    np.testing.assert_array_equal(r["csr_off"], ref["csr_off"])
    np.testing.assert_array_equal(r["csr_ids"], ref["csr_ids"])
    np.testing.assert_array_equal(r["barle_off"], ref["barle_off"])
    np.testing.assert_array_equal(r["barle"], ref["barle"])
    np.testing.assert_array_equal(r["shadow"], O.svf_to_words32(ref["svf"], r["shadow_words"]))


# (format, hour block, accumulation, group size): the plain per-hour path,
# the per-voxel block kernel (group 0), the grouped kernel (1, 2, 4, 8) and
# the shared-memory tile kernel (64).
CASES = ([(fmt, 1, acc, 0) for fmt in (0, 1) for acc in (0, 1, 2)]
         + [(fmt, B, acc, 0) for fmt in (0, 1) for B in (32, 64, 128, 256) for acc in (0, 1, 2)]
         + [(fmt, B, acc, V) for fmt in (0, 1) for V in (4, 8) for B in (32, 64, 128, 256) for acc in (0, 1, 2)
            if not (V == 8 and B == 256)]
         + [(fmt, B, acc, V) for fmt in (0, 1) for V in (1, 2) for B in (64, 128, 256, 512) for acc in (0, 1)]
         + [(fmt, B, acc, 64) for fmt in (0, 1) for B in (64, 128, 256) for acc in (0, 1, 2)]
         + [(fmt, 256, acc, 128) for fmt in (0, 1) for acc in (0, 1, 2)])


@pytest.mark.parametrize("fmt,B,acc,V", CASES)
def test_irradiance_vs_fp64(ctx, scene64, fmt, B, acc, V):
    import torch
    s = scene64
    want = fp64_reference(s)
    out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
    ctx.run_device(s, device_arrays(s), out, neighbor_format=fmt, hour_block=B, accumulation=acc, group_size=V)
    torch.cuda.synchronize()
    e = rel_err(out.cpu().numpy(), want)
    assert e.max() <= REL_TOL, (e.max(), e.mean())


@pytest.mark.parametrize("fmt", [0, 1])
def test_annual_form_vs_fp64(ctx, scene160, fmt):
    import torch
    s = scene160
    want = fp64_reference(s)
    out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
    ctx.run_device(s, device_arrays(s), out, neighbor_format=fmt, reflection=1)
    torch.cuda.synchronize()
    e = rel_err(out.cpu().numpy(), want)
    assert e.max() <= REL_TOL, (e.max(), e.mean())


def test_own_irradiance_without_reflection_vs_fp64(ctx, scene160):
    """reflection=none: each voxel's own direct + diffuse (the FP64 oracle's
    second sum); the reflected share is 1 - own / total."""
    import torch
    from oracle import oracle as O
    s = scene160
    bins, off, ids, sh = oracle_trace(s)
    tot, own = O.annual_fp64(s, sh, off, ids)
    out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
    ctx.run_device(s, device_arrays(s), out, neighbor_format=0, reflection=2)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    e = rel_err(got, own)
    assert e.max() <= REL_TOL, (e.max(), e.mean())
    share = 1.0 - own / tot
    assert share.min() >= 0.0 and share.max() > 0.0   # reflection only adds


@pytest.mark.parametrize("fmt,V", [(0, 0), (1, 0), (0, 8), (1, 8), (1, 4), (0, 1), (1, 2), (0, 64), (1, 64)])
def test_hour_block_vs_fp64_dsm160(ctx, scene160, fmt, V):
    import torch
    s = scene160
    want = fp64_reference(s)
    out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
    ctx.run_device(s, device_arrays(s), out, neighbor_format=fmt, hour_block=128, group_size=V)
    torch.cuda.synchronize()
    e = rel_err(out.cpu().numpy(), want)
    assert e.max() <= REL_TOL, (e.max(), e.mean())


@pytest.mark.parametrize("fmt,acc", [(0, 1), (1, 1), (0, 0), (1, 2)])
def test_tensor_core_kernel_vs_fp64_dsm160(ctx, scene160, fmt, acc):
    """The tcgen05 hour-block kernel (group_size 128: 128-voxel groups, fp16
    slab, split fp16 weights, FP32 accumulation in TMEM) on the 160 x 160
    town: every voxel within 1e-4 of the FP64 oracle, and far closer on
    average."""
    import torch
    s = scene160
    want = fp64_reference(s)
    out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
    ctx.run_device(s, device_arrays(s), out, neighbor_format=fmt, hour_block=256, group_size=128, accumulation=acc)
    torch.cuda.synchronize()
    e = rel_err(out.cpu().numpy(), want)
    assert e.max() <= REL_TOL, (e.max(), e.mean())
    assert e.mean() <= 1e-6, e.mean()


def test_tensor_core_kernel_is_reproducible(ctx, scene160):
    """Entries are scattered into zeroed tiles, so the order in which the
    layout pass stored them does not change the product: runs are
    bit-identical."""
    import torch
    dev = device_arrays(scene160)
    outs = []
    for _ in range(2):
        out = torch.zeros(scene160.num_total, dtype=torch.float32, device="cuda:0")
        ctx.run_device(scene160, dev, out, neighbor_format=0, hour_block=256, group_size=128)
        outs.append(out.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("compressed", [False, True])
def test_drop_in_entry_points(cuda_lib, scene64, compressed):
    """The reference-shaped host entry points (host arrays in, host raster out)."""
    from solargpu_b200 import api
    s = scene64
    out = np.zeros(s.num_total, np.float32)
    fn = api.compressed_gpu_irradiance if compressed else api.uncompressed_gpu_irradiance
    rc = fn(s.grid, s.width, s.height, s.num_total, s.num_top, s.pixel_parent, s.wall_z, s.max_height,
            s.sun, s.direct, s.diffuse, s.slopes, s.aspects, out)
    assert rc == 0
    e = rel_err(out, fp64_reference(s))
    assert e.max() <= REL_TOL, (e.max(), e.mean())


@pytest.mark.parametrize("compressed", [False, True])
def test_drop_in_vs_reference_api(cuda_lib, scene64, compressed):
    """Against the reference API rebuilt for sm_100a (FP32 per-hour sums):
    both sit near the FP64 oracle; ours is the closer one."""
    from oracle import oracle as O
    from solargpu_b200 import api
    if O.ref_gpu() is None:
        pytest.skip("reference CUDA pipeline not built")
    s = scene64
    ref = O.ref_irradiance(s, compressed)
    out = np.zeros(s.num_total, np.float32)
    fn = api.compressed_gpu_irradiance if compressed else api.uncompressed_gpu_irradiance
    fn(s.grid, s.width, s.height, s.num_total, s.num_top, s.pixel_parent, s.wall_z, s.max_height,
       s.sun, s.direct, s.diffuse, s.slopes, s.aspects, out)
    want = fp64_reference(s)
    e_ours, e_ref = rel_err(out, want), rel_err(ref, want)
    assert e_ours.max() <= REL_TOL
    assert rel_err(out, ref.astype(np.float64)).max() <= REL_TOL
    assert e_ours.mean() <= e_ref.mean() * 1.01 + 1e-9


@pytest.mark.parametrize("name", ["dsm64", "dsm160"])
@pytest.mark.parametrize("compressed", [False, True])
def test_drop_in_vs_reference_golden_rasters(cuda_lib, name, compressed):
    """Against the reference API's own annual rasters, made on a B200 and
    committed (tests/golden/ref_annual_<name>.npz): within 1e-4 per voxel."""
    import os
    from conftest import GOLDEN
    from solargpu_b200 import api
    g = np.load(os.path.join(GOLDEN, f"ref_annual_{name}.npz"))
    s = load_scene(name)
    out = np.zeros(s.num_total, np.float32)
    fn = api.compressed_gpu_irradiance if compressed else api.uncompressed_gpu_irradiance
    assert fn(s.grid, s.width, s.height, s.num_total, s.num_top, s.pixel_parent, s.wall_z, s.max_height,
              s.sun, s.direct, s.diffuse, s.slopes, s.aspects, out) == 0
    ref = g["compressed" if compressed else "uncompressed"].astype(np.float64)
    assert rel_err(out, ref).max() <= REL_TOL


def test_cxx_caller_against_reference_header(cuda_lib, scene64, tmp_path):
    """A C++ program compiled against the reference's own API header
    (include/solar_gpu_api.h, oracle/cxx_caller.cpp) calls both mangled entry
    points with std::vector inputs through libsolargpu_b200.so; its rasters
    equal the C entry points' bit for bit."""
    import os
    import subprocess
    from conftest import ROOT
    from solargpu_b200 import api
    exe = os.path.join(ROOT, "oracle", "_ref", "cxx_caller")
    if not os.path.exists(exe):
        pytest.skip("C++ caller not built (needs the reference header at build time)")
    s = scene64
    inp, outp = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(inp, "wb") as f:
        f.write(np.array([s.width, s.height, s.num_total, s.num_top], np.int32).tobytes())
        f.write(np.float32(s.max_height).tobytes())
        for a, dt in ((s.grid, np.float32), (s.pixel_parent, np.int32), (s.wall_z, np.float32),
                      (s.sun, np.float32), (s.direct, np.float32), (s.diffuse, np.float32),
                      (s.slopes, np.float32), (s.aspects, np.float32)):
            f.write(np.ascontiguousarray(a, dt).tobytes())
    subprocess.run([exe, inp, outp], check=True, timeout=600)
    raw = np.fromfile(outp, np.uint8)
    rc = raw[:8].view(np.int32)
    res = raw[8:].view(np.float32).reshape(2, s.num_total)
    assert list(rc) == [0, 0]
    for k, fn in enumerate((api.uncompressed_gpu_irradiance, api.compressed_gpu_irradiance)):
        out = np.zeros(s.num_total, np.float32)
        fn(s.grid, s.width, s.height, s.num_total, s.num_top, s.pixel_parent, s.wall_z, s.max_height,
           s.sun, s.direct, s.diffuse, s.slopes, s.aspects, out)
        assert np.array_equal(res[k], out)


def test_trace_matches_reference_kernel_dsm1024(ctx):
    """The 1024 x 1024 city (1.5 M voxels, the full-scale tracer path: visiting
    order, direction parts, shadow words merged across parts) against the
    reference's own viewshed stage rebuilt for sm_100a: CSR ids, ba-RLE bytes
    and offsets, and the shadow bitmap, bit for bit."""
    from oracle import oracle as O
    from solargpu_b200 import inputs
    if O.ref_gpu() is None:
        pytest.skip("reference CUDA pipeline not built")
    s = inputs.make_scene("dsm1024")
    ref = O.ref_stage1(s)
    r = ctx.trace(s, device_arrays(s))
    np.testing.assert_array_equal(r["csr_off"], ref["csr_off"])
    np.testing.assert_array_equal(r["csr_ids"], ref["csr_ids"])
    np.testing.assert_array_equal(r["barle_off"], ref["barle_off"])
    np.testing.assert_array_equal(r["barle"], ref["barle"])
    np.testing.assert_array_equal(r["shadow"], O.svf_to_words32(ref["svf"], r["shadow_words"]))


def test_grouped_results_are_reproducible(ctx, scene160):
    """Union entries are built in a fixed order, so runs are bit-identical."""
    import torch
    dev = device_arrays(scene160)
    outs = []
    for _ in range(2):
        out = torch.zeros(scene160.num_total, dtype=torch.float32, device="cuda:0")
        ctx.run_device(scene160, dev, out, neighbor_format=1, hour_block=128, group_size=8)
        outs.append(out.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("B", [128, 256])
def test_tiles_equal_per_voxel_lists_on_barle(ctx, scene160, B):
    """The tile kernel applies each voxel's entries in the ba-RLE list order
    with the same FMA chain, so it reproduces group size 1 bit for bit."""
    import torch
    dev = device_arrays(scene160)
    outs = []
    for V in (1, 64, 64):
        out = torch.zeros(scene160.num_total, dtype=torch.float32, device="cuda:0")
        ctx.run_device(scene160, dev, out, neighbor_format=1, hour_block=B, accumulation=1, group_size=V)
        outs.append(out.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[1], outs[2])


@pytest.mark.parametrize("fmt", [0, 1])
def test_run_from_cached_lists_with_new_tmy(ctx, scene160, fmt, tmp_path):
    """Stage 1 saved to disk and re-run with other hourly irradiance gives the
    same raster as a full run on that irradiance."""
    import dataclasses
    import torch
    from solargpu_b200 import cache
    s = scene160
    dev = device_arrays(s)
    p = str(tmp_path / "lists.npz")
    cache.save_lists(p, ctx.trace(s, dev, neighbor_format=fmt), s, fmt=fmt)
    s2 = dataclasses.replace(s, direct=(s.direct * np.float32(0.7)), diffuse=(s.diffuse * np.float32(1.3)))
    want = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
    ctx.run_device(s2, dev, want, neighbor_format=fmt)
    got = torch.zeros_like(want)
    ctx.run_lists(s2, dev, cache.load_lists(p, s2), got)
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), want.cpu().numpy())
    assert rel_err(got.cpu().numpy(), fp64_reference(s2)).max() <= REL_TOL


def test_run_lists_rejects_other_sky_bins(ctx, scene64):
    import torch
    from solargpu_b200 import api
    dev = device_arrays(scene64)
    r = ctx.trace(scene64, dev, neighbor_format=0)
    r["active_bins"] += 1
    out = torch.zeros(scene64.num_total, dtype=torch.float32, device="cuda:0")
    with pytest.raises(api.SolarGPUError) as e:
        ctx.run_lists(scene64, dev, r, out)
    assert e.value.code == -1


def test_invalid_hour_block_for_group_is_rejected(ctx, scene64):
    import torch
    from solargpu_b200 import api
    out = torch.zeros(scene64.num_total, dtype=torch.float32, device="cuda:0")
    with pytest.raises(api.SolarGPUError) as e:
        ctx.run_device(scene64, device_arrays(scene64), out, hour_block=256, group_size=8)
    assert e.value.code == -1


def test_invalid_pixel_parent_is_rejected(ctx, scene64):
    import torch
    from solargpu_b200 import api
    dev = device_arrays(scene64)
    dev["pixel_parent"] = dev["pixel_parent"].clone()
    dev["pixel_parent"][scene64.num_top + 3] = scene64.num_top + 5   # wall parent out of range
    out = torch.zeros(scene64.num_total, dtype=torch.float32, device="cuda:0")
    with pytest.raises(api.SolarGPUError) as e:
        ctx.run_device(scene64, dev, out)
    assert e.value.code == -1
    ctx.run_device(scene64, device_arrays(scene64), out)   # the context stays usable


def _edge_scene(kind):
    """Degenerate scenes: a flat field (no walls, nearly empty lists), a lone
    tower (a few wall voxels with long lists next to many empty ones) and a
    7 x 5 strip whose voxel count is no multiple of 4 or 64."""
    from solargpu_b200 import inputs
    if kind == "flat":
        z = np.zeros((24, 24), np.float32)
    elif kind == "tower":
        z = np.zeros((32, 32), np.float32)
        z[14:17, 14:17] = 25.0
    else:
        z = np.zeros((5, 7), np.float32)
        z[2, 3] = 3.0
    cfg = inputs.DsmConfig(f"edge_{kind}", z.shape[1], 0, 0, seed=5)
    return inputs.make_scene(cfg, heights=z)


@pytest.mark.parametrize("kind", ["flat", "tower", "strip"])
@pytest.mark.parametrize("fmt,B,V", [(0, 256, 64), (1, 256, 64), (0, 128, 64), (1, 128, 1), (0, 1, 0),
                                     (0, 256, 128), (1, 256, 128)])
def test_degenerate_scenes(ctx, kind, fmt, B, V):
    import torch
    s = _edge_scene(kind)
    out = torch.zeros(s.num_total, dtype=torch.float32, device="cuda:0")
    ctx.run_device(s, device_arrays(s), out, neighbor_format=fmt, hour_block=B, group_size=V, accumulation=1)
    torch.cuda.synchronize()
    e = rel_err(out.cpu().numpy(), fp64_reference(s))
    assert e.max() <= REL_TOL, (e.max(), e.mean())
    r = ctx.trace(s, device_arrays(s), neighbor_format=2)
    bins, off, ids, sh = oracle_trace(s)
    assert np.array_equal(r["csr_off"], off) and np.array_equal(r["csr_ids"], ids)
    assert np.array_equal(r["shadow"], sh)
