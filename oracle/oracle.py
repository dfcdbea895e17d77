"""ctypes front end of the CPU oracle (test infrastructure only).

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product package never does.  It wraps

* ``_build/liboracle.so`` -- the C restatement in ``solar_oracle.c``;
* ``_ref/libref_host.so`` -- the reference's own host code (ba-RLE encoder,
  sky bins, voxelization) compiled from its sources, when it was built;
* ``_ref/libsolarref.so`` -- the reference CUDA pipeline rebuilt for sm_100a
  with ``ref_driver.cu``, when it was built (runs only where a GPU exists).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HOURS = 8760
_P = C.c_void_p


def build(ref: str | None = None) -> None:
    """Runs the oracle Makefile (the reference libraries only if `ref` exists)."""
    env = dict(os.environ)
    cmd = ["make", "-s", "-C", HERE]
    if ref is not None:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True, env=env)


_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
    return _LIB


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_P)


# ---------------------------------------------------------------- sky bins

def sky_bins(sun: np.ndarray) -> dict:
    sun = np.ascontiguousarray(sun, np.float32)
    fd = np.zeros(72 * 18, np.int32)
    sdi = np.zeros(HOURS, np.int32)
    nud = np.zeros((HOURS, 2), np.float32)
    meta = np.zeros(5, np.int32)
    lib().orc_sky_bins(_ptr(sun), C.c_float(5.0), C.c_float(5.0), _ptr(fd), _ptr(sdi), _ptr(nud), _ptr(meta))
    return dict(full_to_dense=fd, sun_dense_idx=sdi, nudged=nud, hsize=int(meta[0]),
                vsize=int(meta[1]), vsize_full=int(meta[2]), active=int(meta[3]),
                words8=int(meta[4]), words32=(int(meta[3]) + 31) // 32)


def directions(bins: dict):
    D = bins["hsize"] * bins["vsize_full"]
    dirs = np.zeros((D, 3), np.float32)
    dense = np.zeros(D, np.int32)
    upper = np.zeros(D, np.int32)
    lib().orc_directions(bins["hsize"], bins["vsize"], C.c_float(5.0), C.c_float(5.0),
                         _ptr(bins["full_to_dense"]), _ptr(dirs), _ptr(dense), _ptr(upper))
    return dirs, dense, upper


# ---------------------------------------------------------------- tracer

def trace(scene, bins: dict | None = None, v0: int = 0, v1: int | None = None,
          fma_mode: int = 1, nthreads: int | None = None):
    """DDA trace of voxels [v0, v1).  Returns (off int64 [n+1], ids int32,
    shadow uint32 [n, words32])."""
    if bins is None:
        bins = sky_bins(scene.sun)
    dirs, dense, upper = directions(bins)
    v1 = scene.num_total if v1 is None else v1
    n = v1 - v0
    D = dirs.shape[0]
    w32 = bins["words32"]
    nthreads = nthreads or os.cpu_count() or 1
    out = np.zeros(0, np.int32)
    cnt_all = np.zeros(n, np.int32)
    sh = np.zeros((n, w32), np.uint32)
    chunk = max(1, min(n, (1 << 28) // (D * 4)))
    lists = []
    wall = scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        nb = np.zeros((b - a, D), np.int32)
        cnt = np.zeros(b - a, np.int32)
        lib().orc_trace(_ptr(scene.grid), scene.width, scene.height, scene.num_total, scene.num_top,
                        _ptr(scene.pixel_parent), _ptr(wall), C.c_float(scene.max_height),
                        _ptr(dirs), _ptr(dense), _ptr(upper), D, v0 + a, v0 + b,
                        _ptr(nb), _ptr(cnt), sh[a:b].ctypes.data_as(_P), w32, fma_mode, nthreads)
        cnt_all[a:b] = cnt
        mask = np.arange(D)[None, :] < cnt[:, None]
        lists.append(nb[mask])
    out = np.concatenate(lists) if lists else out
    off = np.zeros(n + 1, np.int64)
    np.cumsum(cnt_all, out=off[1:])
    return off, out.astype(np.int32), sh


def trace_list(scene, voxels: np.ndarray, bins: dict | None = None, lists: bool = True,
               nthreads: int | None = None):
    """DDA trace of an arbitrary voxel list (any order), each voxel exactly as
    `trace` traces it.  Returns (off int64 [n+1], ids int32, shadow uint32
    [n, words32]); with lists=False only the shadow words are kept (off and
    ids are None), which needs no [n][D] buffer."""
    if bins is None:
        bins = sky_bins(scene.sun)
    dirs, dense, upper = directions(bins)
    vox = np.ascontiguousarray(voxels, np.int32)
    n = vox.size
    D = dirs.shape[0]
    w32 = bins["words32"]
    nthreads = nthreads or os.cpu_count() or 1
    sh = np.zeros((n, w32), np.uint32)
    wall = scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)
    args = (_ptr(scene.grid), scene.width, scene.height, scene.num_total, scene.num_top,
            _ptr(scene.pixel_parent), _ptr(wall), C.c_float(scene.max_height), _ptr(dirs), _ptr(dense),
            _ptr(upper), D)
    if not lists:
        rc = lib().orc_trace_list(*args, _ptr(vox), n, None, None, sh.ctypes.data_as(_P), w32, 1, nthreads)
        if rc != 0:
            raise ValueError("voxel index out of range")
        return None, None, sh
    chunk = max(1, min(n, (1 << 28) // (D * 4)))
    cnt_all = np.zeros(n, np.int32)
    out = []
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        nb = np.zeros((b - a, D), np.int32)
        cnt = np.zeros(b - a, np.int32)
        rc = lib().orc_trace_list(*args, _ptr(vox[a:b]), b - a, _ptr(nb), _ptr(cnt), sh[a:b].ctypes.data_as(_P),
                                  w32, 1, nthreads)
        if rc != 0:
            raise ValueError("voxel index out of range")
        cnt_all[a:b] = cnt
        out.append(nb[np.arange(D)[None, :] < cnt[:, None]])
    off = np.zeros(n + 1, np.int64)
    np.cumsum(cnt_all, out=off[1:])
    ids = np.concatenate(out).astype(np.int32) if out else np.zeros(0, np.int32)
    return off, ids, sh


def trace_one(grid: np.ndarray, maxz: float, gx: int, gy: int, base_z: float, c, is_upper: bool,
              fma_mode: int = 1) -> int:
    """One DDA ray over a bare heightmap grid [H][W] from cell (gx, gy) at
    base_z along c = (cx, cy, cz); the 1-based hit cell id or 0."""
    g = np.ascontiguousarray(grid, np.float32)
    H, W = g.shape
    f = lib().orc_trace_one
    f.restype = C.c_int
    f.argtypes = [_P, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                  C.c_int, C.c_int]
    return f(_ptr(g), W, H, float(maxz), int(gx), int(gy), float(base_z), float(np.float32(c[0])),
             float(np.float32(c[1])), float(np.float32(c[2])), int(bool(is_upper)), int(fma_mode))


def trace_steps(scene, voxels: np.ndarray, bins: dict | None = None) -> np.ndarray:
    """DDA steps of every ray of the listed voxels: int16 [n][D] (saturating
    at 32767); a step is one move to the next cell (the loop of
    viewshed_kernels.cu:31-58)."""
    if bins is None:
        bins = sky_bins(scene.sun)
    dirs, dense, upper = directions(bins)
    vox = np.ascontiguousarray(voxels, np.int32)
    D = dirs.shape[0]
    steps = np.zeros((vox.size, D), np.int16)
    wall = scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)
    lib().orc_trace_steps(_ptr(scene.grid), scene.width, scene.height, scene.num_total, scene.num_top,
                          _ptr(scene.pixel_parent), _ptr(wall), C.c_float(scene.max_height), _ptr(dirs),
                          _ptr(dense), _ptr(upper), D, _ptr(vox), vox.size, steps.ctypes.data_as(_P))
    return steps


# ---------------------------------------------------------------- ba-RLE

def barle_encode(ids) -> bytes:
    ids = np.ascontiguousarray(ids, np.int32)
    cap = 8 * max(1, ids.size) + 64
    out = np.zeros(cap, np.uint8)
    n = lib().orc_barle_encode(_ptr(ids), ids.size, _ptr(out), cap)
    if n < 0:
        raise RuntimeError("encode overflow")
    return out[:n].tobytes()


def barle_encode_csr(off: np.ndarray, ids: np.ndarray):
    """Encodes every list; returns (byte offsets int64 [n+1], bytes uint8)."""
    off = np.ascontiguousarray(off, np.int64)
    ids = np.ascontiguousarray(ids, np.int32)
    n = off.size - 1
    sizes = np.zeros(n, np.int64)
    f = lib().orc_barle_encode_csr
    f.restype = C.c_longlong
    total = f(_ptr(off), _ptr(ids if ids.size else np.zeros(1, np.int32)), n, _ptr(sizes), None, C.c_longlong(0))
    buf = np.zeros(max(1, total), np.uint8)
    f(_ptr(off), _ptr(ids if ids.size else np.zeros(1, np.int32)), n, _ptr(sizes), _ptr(buf), C.c_longlong(buf.size))
    boff = np.zeros(n + 1, np.int64)
    np.cumsum(sizes, out=boff[1:])
    return boff, buf[:total]


def barle_decode(data: bytes) -> np.ndarray:
    arr = np.frombuffer(data, np.uint8).copy() if len(data) else np.zeros(1, np.uint8)
    cap = 2 * len(data) + 16
    out = np.zeros(cap, np.uint32)
    n = lib().orc_barle_decode(_ptr(arr), len(data), _ptr(out), cap)
    if n < 0:
        raise ValueError(f"malformed ba-RLE stream ({n})")
    return out[:n]


# ---------------------------------------------------------------- FP64 irradiance

def annual_fp64(scene, shadow: np.ndarray, off: np.ndarray, ids: np.ndarray, nthreads: int | None = None):
    """FP64 annual irradiance (Wh/m^2) per voxel, annual-sum form.  Returns
    (total, direct_plus_diffuse)."""
    out = np.zeros(scene.num_total, np.float64)
    dd = np.zeros(scene.num_total, np.float64)
    wall = scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)
    sh = np.ascontiguousarray(shadow, np.uint32)
    lib().orc_annual_fp64(_ptr(scene.grid), scene.width, scene.height, scene.num_total, scene.num_top,
                          _ptr(scene.pixel_parent), _ptr(wall), _ptr(scene.slopes), _ptr(scene.aspects),
                          _ptr(scene.sun), _ptr(scene.direct), _ptr(scene.diffuse),
                          _ptr(sh), sh.shape[1], _ptr(np.ascontiguousarray(off, np.int64)),
                          _ptr(np.ascontiguousarray(ids, np.int32) if ids.size else np.zeros(1, np.int32)),
                          _ptr(out), _ptr(dd), nthreads or os.cpu_count() or 1)
    return out, dd


def annual_fp64_sample(scene, sample, off, ids, shadow, cells, cell_shadow, nthreads=None) -> np.ndarray:
    """FP64 annual irradiance (annual-sum form, as `annual_fp64`) of the
    voxels `sample`, from their lists (off [n+1] from 0, ids 1-based cells)
    and shadow words, given the shadow words of every top cell the lists name
    (`cells`, ascending, 0-based)."""
    sample = np.ascontiguousarray(sample, np.int32)
    cells = np.ascontiguousarray(cells, np.int32)
    sh = np.ascontiguousarray(shadow, np.uint32)
    csh = np.ascontiguousarray(cell_shadow, np.uint32)
    out = np.zeros(sample.size, np.float64)
    wall = scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)
    ids = np.ascontiguousarray(ids, np.int32)
    nh = lib().orc_annual_fp64_sample(
        _ptr(scene.grid), scene.width, scene.height, scene.num_total, scene.num_top,
        _ptr(scene.pixel_parent), _ptr(wall), _ptr(scene.slopes), _ptr(scene.aspects),
        _ptr(np.ascontiguousarray(scene.sun, np.float32)), _ptr(scene.direct), _ptr(scene.diffuse),
        _ptr(sample), sample.size, _ptr(sh), _ptr(np.ascontiguousarray(off, np.int64)),
        _ptr(ids if ids.size else np.zeros(1, np.int32)), _ptr(cells if cells.size else np.zeros(1, np.int32)),
        cells.size, _ptr(csh if csh.size else np.zeros((1, sh.shape[1]), np.uint32)), sh.shape[1],
        _ptr(out), nthreads or os.cpu_count() or 1)
    if nh < 0:
        raise ValueError("a list names a cell that is not in `cells`")
    return out


def sample_reference(scene, sample: np.ndarray, nthreads: int | None = None) -> dict:
    """Everything the oracle needs to check a voxel sample of a scene too large
    for a full CPU pass: the sample's own Stage 1 (lists + shadow words),
    Stage 1 shadow words of every top cell its lists name, and the FP64 annual
    irradiance of the sample from those oracle-built products."""
    import time
    bins = sky_bins(scene.sun)
    t0 = time.perf_counter()
    off, ids, sh = trace_list(scene, sample, bins, nthreads=nthreads)
    cells = np.unique(ids.astype(np.int64) - 1).astype(np.int32)
    _, _, csh = trace_list(scene, cells, bins, lists=False, nthreads=nthreads)
    t1 = time.perf_counter()
    tot = annual_fp64_sample(scene, sample, off, ids, sh, cells, csh, nthreads=nthreads)
    t2 = time.perf_counter()
    return dict(off=off, ids=ids, shadow=sh, cells=cells, cell_shadow=csh, annual=tot, bins=bins,
                trace_s=t1 - t0, irradiance_s=t2 - t1)


def hourly_fp64(scene, shadow, off, ids, v0=0, v1=None, hblock=64, nthreads=None):
    """FP64 per-hour method for voxels [v0, v1) (the CPU baseline's method)."""
    v1 = scene.num_total if v1 is None else v1
    out = np.zeros(v1 - v0, np.float64)
    wall = scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)
    sh = np.ascontiguousarray(shadow, np.uint32)
    lib().orc_hourly_fp64(_ptr(scene.grid), scene.width, scene.height, scene.num_total, scene.num_top,
                          _ptr(scene.pixel_parent), _ptr(wall), _ptr(scene.slopes), _ptr(scene.aspects),
                          _ptr(scene.sun), _ptr(scene.direct), _ptr(scene.diffuse),
                          _ptr(sh), sh.shape[1], _ptr(np.ascontiguousarray(off, np.int64)),
                          _ptr(np.ascontiguousarray(ids, np.int32) if ids.size else np.zeros(1, np.int32)),
                          v0, v1, hblock, _ptr(out), nthreads or os.cpu_count() or 1)
    return out


def hour_table(sun, dni, dhi) -> np.ndarray:
    out = np.zeros((HOURS, 11), np.float64)
    n = lib().orc_hour_table_dump(_ptr(np.ascontiguousarray(sun, np.float32)),
                                  _ptr(np.ascontiguousarray(dni, np.float32)),
                                  _ptr(np.ascontiguousarray(dhi, np.float32)), _ptr(out))
    return out[:n]


# ---------------------------------------------------------------- reference builds

def ref_host():
    """The reference's own host code, or None when it was not built."""
    path = os.path.join(HERE, "_ref", "libref_host.so")
    return C.CDLL(path) if os.path.exists(path) else None


def ref_barle_compress(ids) -> bytes:
    L = ref_host()
    ids = np.ascontiguousarray(ids, np.int32)
    raw = np.concatenate([ids, np.zeros(1, np.int32)])
    cap = 8 * max(1, ids.size) + 64
    out = np.zeros(cap, np.uint8)
    n = L.ref_barle_compress(_ptr(raw), raw.size, _ptr(out), cap)
    return out[:n].tobytes()


def ref_sky_bins(sun) -> dict:
    L = ref_host()
    sun = np.ascontiguousarray(sun, np.float32)
    fd = np.zeros(72 * 18, np.int32)
    sdi = np.zeros(HOURS, np.int32)
    nud = np.zeros((HOURS, 2), np.float32)
    meta = np.zeros(5, np.int32)
    L.ref_sky_bins(_ptr(sun), _ptr(fd), _ptr(sdi), _ptr(nud), _ptr(meta))
    return dict(full_to_dense=fd, sun_dense_idx=sdi, nudged=nud, hsize=int(meta[0]),
                vsize=int(meta[1]), vsize_full=int(meta[2]), active=int(meta[3]), words8=int(meta[4]))


def ref_voxelize(heights: np.ndarray):
    L = ref_host()
    h = np.ascontiguousarray(heights, np.float32)
    H, W = h.shape
    cap = 64 * W * H
    par = np.zeros(cap, np.int32)
    z = np.zeros(cap, np.float32)
    asp = np.zeros(cap, np.float32)
    n = L.ref_detect_walls(_ptr(h), W, H, C.c_float(1.0), _ptr(par), _ptr(z), _ptr(asp), cap)
    sl = np.zeros(W * H, np.float32)
    ta = np.zeros(W * H, np.float32)
    L.ref_top_slope_aspect(_ptr(h), W, H, C.c_float(1.0), _ptr(sl), _ptr(ta))
    return par[:n], z[:n], asp[:n], sl, ta


def ref_sun_positions(lon: float, lat: float, tz: int) -> np.ndarray:
    L = ref_host()
    out = np.zeros((8784, 2), np.float32)
    n = L.ref_sun_positions(C.c_float(lon), C.c_float(lat), tz, _ptr(out), 8784)
    return out[:n]


class _RefStage1(C.Structure):
    _fields_ = [("num_total", C.c_longlong), ("nnz", C.c_longlong),
                ("csr_off", C.POINTER(C.c_int)), ("csr_ids", C.POINTER(C.c_int)),
                ("barle_bytes", C.c_longlong), ("barle_off", C.POINTER(C.c_int)),
                ("barle", C.POINTER(C.c_ubyte)), ("svf_words8", C.c_int),
                ("svf", C.POINTER(C.c_ubyte))]


def ref_gpu():
    """The reference CUDA pipeline library, or None when it was not built."""
    path = os.path.join(HERE, "_ref", "libsolarref.so")
    return C.CDLL(path) if os.path.exists(path) else None


def ref_stage1(scene) -> dict:
    """Runs the reference's own viewshed stage on the GPU; returns its CSR
    lists, ba-RLE streams and shadow bitmap (reference layout)."""
    L = ref_gpu()
    st = _RefStage1()
    wall = scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)
    rc = L.ref_stage1(_ptr(scene.grid), scene.width, scene.height, scene.num_total, scene.num_top,
                      _ptr(scene.pixel_parent), _ptr(wall), C.c_float(scene.max_height),
                      _ptr(np.ascontiguousarray(scene.sun, np.float32)), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"ref_stage1 failed: {rc}")
    n = int(st.num_total)
    out = dict(
        csr_off=np.ctypeslib.as_array(st.csr_off, (n + 1,)).astype(np.int64),
        csr_ids=np.ctypeslib.as_array(st.csr_ids, (max(1, st.nnz),))[:st.nnz].copy(),
        barle_off=np.ctypeslib.as_array(st.barle_off, (n + 1,)).astype(np.int64),
        barle=np.ctypeslib.as_array(st.barle, (max(1, st.barle_bytes),))[:st.barle_bytes].copy(),
        svf=np.ctypeslib.as_array(st.svf, (st.svf_words8 * n,)).reshape(st.svf_words8, n).copy(),
    )
    L.ref_stage1_free(C.byref(st))
    return out


def ref_irradiance(scene, compressed: bool) -> np.ndarray:
    """Runs the stock reference API (uncompressed or compressed) on the GPU."""
    L = ref_gpu()
    out = np.zeros(scene.num_total, np.float32)
    wall = scene.wall_z if scene.wall_z.size else None
    fn = L.ref_compressed if compressed else L.ref_uncompressed
    rc = fn(_ptr(scene.grid), scene.width, scene.height, scene.num_total, scene.num_top,
            _ptr(scene.pixel_parent), _ptr(wall), C.c_float(scene.max_height),
            _ptr(np.ascontiguousarray(scene.sun, np.float32)), _ptr(scene.direct), _ptr(scene.diffuse),
            _ptr(scene.slopes), _ptr(scene.aspects), _ptr(out))
    if rc != 0:
        raise RuntimeError(f"reference API returned {rc}")
    return out


def svf_to_words32(svf8: np.ndarray, words32: int) -> np.ndarray:
    """Converts the reference shadow layout (uint8 [words8][N], word-major /
    voxel-minor, include/voxel_types.h:36-50) to uint32 [N][words32]."""
    w8, n = svf8.shape
    pad = np.zeros((words32 * 4, n), np.uint8)
    pad[:w8] = svf8
    b = pad.T.reshape(n, words32, 4).astype(np.uint32)
    return (b[..., 0] | (b[..., 1] << 8) | (b[..., 2] << 16) | (b[..., 3] << 24)).astype(np.uint32)


def cpu_sample(scene, sample: np.ndarray, hblock: int = 64, nthreads: int | None = None) -> dict:
    """Times the FP64 per-hour method on a bounded sample (see orc_cpu_sample)
    and scales it to the whole scene.  Returns seconds per stage and the
    estimated whole-scene voxel-hours/s."""
    sample = np.ascontiguousarray(sample, np.int32)
    times = np.zeros(3, np.float64)
    wall = scene.wall_z if scene.wall_z.size else np.zeros(1, np.float32)
    nthreads = nthreads or os.cpu_count() or 1
    nh = lib().orc_cpu_sample(_ptr(scene.grid), scene.width, scene.height, scene.num_total, scene.num_top,
                              _ptr(scene.pixel_parent), _ptr(wall), C.c_float(scene.max_height),
                              _ptr(scene.slopes), _ptr(scene.aspects), _ptr(np.ascontiguousarray(scene.sun, np.float32)),
                              _ptr(scene.direct), _ptr(scene.diffuse), _ptr(sample), sample.size, hblock, nthreads,
                              _ptr(times))
    ns = sample.size
    hb = min(hblock, nh)
    blocks = nh / hb
    t_full = times[0] / ns * scene.num_total + (times[1] + times[2] / ns * scene.num_total) * blocks
    return dict(trace_s=float(times[0]), table_s=float(times[1]), sums_s=float(times[2]), hours=int(nh),
                hblock=int(hb), threads=int(nthreads), est_full_s=float(t_full),
                voxel_hours_per_s=float(scene.num_total * nh / t_full))
