"""Python front end of libsolargpu_b200.so (ctypes over the C ABI in
include/solargpu_b200.h).

``uncompressed_gpu_irradiance`` / ``compressed_gpu_irradiance`` mirror the
reference entry points (include/solar_gpu_api.h:37-54) argument for
argument: host arrays in, the annual irradiance written into
``irradiance_out``, 0 returned on success.  Where the reference would exit
the process on a CUDA error, these raise :class:`SolarGPUError`.

:class:`Context` exposes the rest of the ABI: device-resident runs on a
caller stream, Stage 1 results for parity checks, stage timings.

The library is the only compute path: if it is missing or no GPU is
present, calls raise; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsolargpu_b200.so")
HOURS_PER_YEAR = 8760

CSR, BARLE, BOTH = 0, 1, 2
ACC_FP64, ACC_KAHAN, ACC_FP32 = 0, 1, 2
REFL_HOURLY, REFL_ANNUAL, REFL_NONE = 0, 1, 2

_ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "no CUDA device",
           -4: "out of device memory", -5: "device data check failed"}


class SolarGPUError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [("neighbor_format", C.c_int), ("hour_block", C.c_int), ("accumulation", C.c_int),
                ("reflection", C.c_int), ("chunk_voxels", C.c_longlong), ("use_graph", C.c_int),
                ("time_kernels", C.c_int), ("group_size", C.c_int)]


class SceneDesc(C.Structure):
    _fields_ = [("grid", C.c_void_p), ("grid_width", C.c_int), ("grid_height", C.c_int),
                ("num_total_voxels", C.c_int), ("num_top_voxels", C.c_int),
                ("pixel_parent", C.c_void_p), ("wall_z", C.c_void_p), ("max_height", C.c_float),
                ("sun_positions", C.c_void_p), ("direct_irradiance", C.c_void_p),
                ("diffuse_irradiance", C.c_void_p), ("slopes", C.c_void_p), ("aspects", C.c_void_p)]


class ListsDesc(C.Structure):
    _fields_ = [("format", C.c_int), ("offsets", C.c_void_p), ("data", C.c_void_p), ("data_size", C.c_longlong),
                ("shadow", C.c_void_p), ("shadow_words", C.c_int), ("active_bins", C.c_int)]


_LIB = None


def lib() -> C.CDLL:
    """Loads the CUDA library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise SolarGPUError(-3, f"{LIB_PATH} is missing; build it with `python -m solargpu_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i, f, ll = C.c_void_p, C.c_int, C.c_float, C.c_longlong
        L.solar_gpu_last_error.restype = C.c_char_p
        L.solar_gpu_last_launch_count.restype = ll
        L.solar_gpu_last_launch_count.argtypes = [vp]
        L.solar_gpu_last_reflection_entries.restype = ll
        L.solar_gpu_last_reflection_entries.argtypes = [vp]
        L.solar_gpu_last_staged_rows.restype = ll
        L.solar_gpu_last_staged_rows.argtypes = [vp]
        L.solar_gpu_last_weighted_entries.restype = ll
        L.solar_gpu_last_weighted_entries.argtypes = [vp]
        for name in ("solar_gpu_uncompressed_gpu_irradiance", "solar_gpu_compressed_gpu_irradiance"):
            fn = getattr(L, name)
            fn.argtypes = [vp, i, i, i, i, vp, vp, f, vp, i, vp, i, vp, i, vp, vp, vp]
            fn.restype = i
        L.solar_gpu_create.argtypes = [i, C.POINTER(vp)]
        L.solar_gpu_destroy.argtypes = [vp]
        L.solar_gpu_destroy.restype = None
        L.solar_gpu_release.argtypes = [vp]
        L.solar_gpu_set_memory_limit.argtypes = [vp, C.c_longlong]
        L.solar_gpu_memory_held.argtypes = [vp]
        L.solar_gpu_memory_held.restype = C.c_longlong
        L.solar_gpu_default_options.argtypes = [C.POINTER(Options)]
        L.solar_gpu_default_options.restype = None
        L.solar_gpu_run_host.argtypes = [vp, C.POINTER(Options), C.POINTER(SceneDesc), vp]
        L.solar_gpu_run_device.argtypes = [vp, C.POINTER(Options), C.POINTER(SceneDesc), vp, vp]
        L.solar_gpu_trace.argtypes = [vp, C.POINTER(Options), C.POINTER(SceneDesc), vp]
        L.solar_gpu_trace_sizes.argtypes = [vp, C.POINTER(ll), C.POINTER(ll), C.POINTER(i), C.POINTER(i), C.POINTER(i)]
        L.solar_gpu_trace_copy.argtypes = [vp, vp, vp, vp, vp, vp]
        L.solar_gpu_trace_copy_range.argtypes = [vp, i, i, vp, vp, vp, vp, vp]
        L.solar_gpu_run_lists.argtypes = [vp, C.POINTER(Options), C.POINTER(SceneDesc), C.POINTER(ListsDesc), vp, vp]
        L.solar_gpu_voxelize.argtypes = [vp, vp, i, i, f, C.POINTER(ll), vp, vp, vp, vp, ll, vp]
        L.solar_gpu_run_batch.argtypes = [C.POINTER(vp), i, C.POINTER(Options), C.POINTER(SceneDesc), C.POINTER(vp), vp]
        L.solar_gpu_gemm_bf16.argtypes = [vp, vp, vp, vp, vp, i, i, i, i, vp]
        L.solar_gpu_last_timings.argtypes = [vp, C.POINTER(C.c_double), i]
        L.solar_gpu_kernel_times.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(ll), i]
        _LIB = L
    return _LIB


def _check(rc: int) -> int:
    if rc != 0:
        raise SolarGPUError(rc, lib().solar_gpu_last_error().decode(errors="replace"))
    return rc


def _host(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a) -> int | None:
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a)


def options(**kw) -> Options:
    o = Options()
    lib().solar_gpu_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


# ---------------------------------------------------------------- drop-in mirror

def _drop_in(compressed, grid_data, grid_width, grid_height, num_total_voxels, num_top_voxels,
             pixel_parent, wall_z, max_height, sun_positions, direct_irradiance, diffuse_irradiance,
             slopes, aspects, irradiance_out):
    grid = _host(grid_data, np.float32)
    pp = _host(pixel_parent, np.int32)
    wz = None if wall_z is None or np.size(wall_z) == 0 else _host(wall_z, np.float32)
    sun = _host(sun_positions, np.float32).reshape(-1, 2)
    dn = _host(direct_irradiance, np.float32)
    df = _host(diffuse_irradiance, np.float32)
    sl = _host(slopes, np.float32)
    asp = _host(aspects, np.float32)
    if not (isinstance(irradiance_out, np.ndarray) and irradiance_out.dtype == np.float32
            and irradiance_out.flags.c_contiguous and irradiance_out.size >= num_total_voxels):
        raise TypeError("irradiance_out must be a contiguous float32 array of num_total_voxels")
    fn = lib().solar_gpu_compressed_gpu_irradiance if compressed else lib().solar_gpu_uncompressed_gpu_irradiance
    return _check(fn(_p(grid), grid_width, grid_height, num_total_voxels, num_top_voxels, _p(pp), _p(wz),
                     float(max_height), _p(sun), sun.shape[0], _p(dn), dn.size, _p(df), df.size,
                     _p(sl), _p(asp), _p(irradiance_out)))


def uncompressed_gpu_irradiance(grid_data, grid_width, grid_height, num_total_voxels, num_top_voxels,
                                pixel_parent, wall_z, max_height, sun_positions, direct_irradiance,
                                diffuse_irradiance, slopes, aspects, irradiance_out) -> int:
    """Annual irradiance with CSR neighbor lists (include/solar_gpu_api.h:37-42)."""
    return _drop_in(False, grid_data, grid_width, grid_height, num_total_voxels, num_top_voxels,
                    pixel_parent, wall_z, max_height, sun_positions, direct_irradiance,
                    diffuse_irradiance, slopes, aspects, irradiance_out)


def compressed_gpu_irradiance(grid_data, grid_width, grid_height, num_total_voxels, num_top_voxels,
                              pixel_parent, wall_z, max_height, sun_positions, direct_irradiance,
                              diffuse_irradiance, slopes, aspects, irradiance_out) -> int:
    """Annual irradiance with ba-RLE neighbor lists decoded on the fly
    (include/solar_gpu_api.h:49-54)."""
    return _drop_in(True, grid_data, grid_width, grid_height, num_total_voxels, num_top_voxels,
                    pixel_parent, wall_z, max_height, sun_positions, direct_irradiance,
                    diffuse_irradiance, slopes, aspects, irradiance_out)


# ---------------------------------------------------------------- context

def run_batch(contexts: list, scenes: list, devs: list, outs: list, stream=None, per_tile: list | None = None,
              **opts) -> None:
    """Runs many scenes (uneven DSM tiles) at once (solar_gpu_run_batch):
    Stage 1 and the list builds tile by tile, then every tile's hour-block
    loop as a branch of one CUDA graph.  One Context per tile; `devs` holds
    each scene's device arrays (as for Context.run_device), `outs` its
    device output; `per_tile` optional per-scene option dicts (over `opts`)."""
    n = len(scenes)
    if not (len(contexts) == len(devs) == len(outs) == n) or n == 0:
        raise ValueError("one context, device-array dict and output per scene")
    o = (Options * n)()
    for i in range(n):
        o[i] = options(**dict(opts, **(per_tile[i] if per_tile else {})))
    descs = (SceneDesc * n)()
    keep = []
    for i, (sc, d) in enumerate(zip(scenes, devs)):
        desc, k = _scene_desc(sc, d)
        descs[i] = desc
        keep.append(k)
    ctx_arr = (C.c_void_p * n)(*[c.h.value for c in contexts])
    out_arr = (C.c_void_p * n)(*[_p(x) for x in outs])
    _check(lib().solar_gpu_run_batch(ctx_arr, n, o, descs, out_arr, stream))


def gemm_bf16(A, B, out=None, out_bf16=None, bias=None, relu: bool = False, stream=None):
    """C = A @ B.T (+ bias, ReLU) on the tensor cores; A [M, K], B [N, K]
    bf16 CUDA tensors (contiguous), M a multiple of 128, N and K of 64."""
    import torch
    M, K = A.shape
    N = B.shape[0]
    if out is None and out_bf16 is None:
        out = torch.empty(M, N, dtype=torch.float32, device=A.device)
    _check(lib().solar_gpu_gemm_bf16(_p(A), _p(B), _p(out), _p(out_bf16), _p(bias), M, N, K, int(relu), stream))
    return out if out is not None else out_bf16


def _scene_desc(scene, dev: dict | None = None) -> tuple[SceneDesc, list]:
    """Builds the C scene struct.  With `dev`, the per-voxel arrays come from
    device tensors (dict with grid, pixel_parent, wall_z, slopes, aspects)."""
    keep = []
    d = SceneDesc()
    d.grid_width = scene.width
    d.grid_height = scene.height
    d.num_total_voxels = scene.num_total
    d.num_top_voxels = scene.num_top
    d.max_height = scene.max_height
    for name, dt in (("sun", np.float32), ("direct", np.float32), ("diffuse", np.float32)):
        a = _host(getattr(scene, name), dt)
        keep.append(a)
    d.sun_positions, d.direct_irradiance, d.diffuse_irradiance = (_p(a) for a in keep[-3:])
    src = dev if dev is not None else {
        "grid": _host(scene.grid, np.float32), "pixel_parent": _host(scene.pixel_parent, np.int32),
        "wall_z": _host(scene.wall_z, np.float32) if scene.wall_z.size else None,
        "slopes": _host(scene.slopes, np.float32), "aspects": _host(scene.aspects, np.float32)}
    keep.append(src)
    d.grid = _p(src["grid"])
    d.pixel_parent = _p(src["pixel_parent"])
    wz = src.get("wall_z")
    d.wall_z = _p(wz) if wz is not None and (getattr(wz, "numel", lambda: np.size(wz))() > 0) else None
    d.slopes = _p(src["slopes"])
    d.aspects = _p(src["aspects"])
    return d, keep


class Context:
    """A device workspace + stream (solar_gpu_create / solar_gpu_destroy)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().solar_gpu_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().solar_gpu_destroy(self.h)
            self.h = C.c_void_p()

    def release(self):
        """Frees the device buffers kept between calls (solar_gpu_release)."""
        _check(lib().solar_gpu_release(self.h))

    def set_memory_limit(self, nbytes: int):
        """Caps the device bytes this context's buffers may hold (0: no cap);
        a call that would pass it raises SolarGPUError (SOLAR_GPU_ERR_OOM)."""
        _check(lib().solar_gpu_set_memory_limit(self.h, int(nbytes)))

    def memory_held(self) -> int:
        return int(lib().solar_gpu_memory_held(self.h))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_host(self, scene, out: np.ndarray | None = None, **opts) -> np.ndarray:
        """Host arrays in and out (copies and read-back inside the call)."""
        o = options(**opts)
        d, keep = _scene_desc(scene)
        if out is None:
            out = np.zeros(scene.num_total, np.float32)
        _check(lib().solar_gpu_run_host(self.h, C.byref(o), C.byref(d), _p(out)))
        return out

    def run_device(self, scene, dev: dict, out, stream=None, **opts) -> None:
        """Device-resident arrays (`dev`, e.g. torch CUDA tensors) and output."""
        o = options(**opts)
        d, keep = _scene_desc(scene, dev)
        _check(lib().solar_gpu_run_device(self.h, C.byref(o), C.byref(d), _p(out), stream))

    def run_lists(self, scene, dev: dict, lists: dict, out, stream=None, **opts) -> None:
        """Stage 2/3 over saved Stage 1 products (`lists`: a `trace()` result
        or `cache.load_lists()`), scene arrays on the device as for
        run_device.  The list format is the one `lists` holds (CSR first)."""
        o = options(**opts)
        d, keep = _scene_desc(scene, dev)
        if "csr_off" in lists:
            fmt, off, data = CSR, _host(lists["csr_off"], np.int64), _host(lists["csr_ids"], np.int32)
        else:
            fmt, off, data = BARLE, _host(lists["barle_off"], np.int64), _host(lists["barle"], np.uint8)
        shadow = _host(lists["shadow"], np.uint32)
        ld = ListsDesc(fmt, _p(off), _p(data) if data.size else None, int(data.size), _p(shadow),
                       int(lists["shadow_words"]), int(lists["active_bins"]))
        _check(lib().solar_gpu_run_lists(self.h, C.byref(o), C.byref(d), C.byref(ld), _p(out), stream))

    def voxelize(self, grid, width: int, height: int, voxel_size: float = 1.0, stream=None) -> dict:
        """Voxelizes a device heightmap (torch tensor [H*W] float32) on the GPU
        (solar_gpu_voxelize); returns device tensors pixel_parent, wall_z,
        slopes, aspects and the counts, packed as the drop-in entry points take
        them."""
        import torch
        n = C.c_longlong()
        _check(lib().solar_gpu_voxelize(self.h, _p(grid), width, height, float(voxel_size), C.byref(n), None, None,
                                        None, None, 0, stream))
        N, T = int(n.value), width * height
        dev = grid.device
        out = {"pixel_parent": torch.empty(N, dtype=torch.int32, device=dev),
               "wall_z": torch.empty(max(1, N - T), dtype=torch.float32, device=dev),
               "slopes": torch.empty(N, dtype=torch.float32, device=dev),
               "aspects": torch.empty(N, dtype=torch.float32, device=dev)}
        _check(lib().solar_gpu_voxelize(self.h, _p(grid), width, height, float(voxel_size), C.byref(n),
                                        _p(out["pixel_parent"]), _p(out["wall_z"]), _p(out["slopes"]),
                                        _p(out["aspects"]), N, stream))
        out["num_total"], out["num_top"] = N, T
        return out

    def stage1(self, scene, dev: dict, neighbor_format: int = BOTH, stream=None, **opts) -> None:
        """Runs Stage 1 only and keeps its products on the device (read them
        with `trace_range`)."""
        o = options(neighbor_format=neighbor_format, **opts)
        d, keep = _scene_desc(scene, dev)
        _check(lib().solar_gpu_trace(self.h, C.byref(o), C.byref(d), stream))

    def trace(self, scene, dev: dict, neighbor_format: int = BOTH, stream=None, **opts) -> dict:
        """Runs Stage 1 and returns its lists and shadow words as numpy arrays."""
        o = options(neighbor_format=neighbor_format, **opts)
        d, keep = _scene_desc(scene, dev)
        _check(lib().solar_gpu_trace(self.h, C.byref(o), C.byref(d), stream))
        ne, nb = C.c_longlong(), C.c_longlong()
        w, a, n = C.c_int(), C.c_int(), C.c_int()
        _check(lib().solar_gpu_trace_sizes(self.h, C.byref(ne), C.byref(nb), C.byref(w), C.byref(a), C.byref(n)))
        N = n.value
        res = {"shadow_words": w.value, "active_bins": a.value}
        csr_off = csr_ids = b_off = b_bytes = None
        if ne.value >= 0:
            csr_off = np.zeros(N + 1, np.int64)
            csr_ids = np.zeros(max(1, ne.value), np.int32)
        if nb.value >= 0:
            b_off = np.zeros(N + 1, np.int64)
            b_bytes = np.zeros(max(1, nb.value), np.uint8)
        shadow = np.zeros((N, w.value), np.uint32)
        _check(lib().solar_gpu_trace_copy(self.h, _p(csr_off), _p(csr_ids), _p(b_off), _p(b_bytes), _p(shadow)))
        if csr_off is not None:
            res["csr_off"], res["csr_ids"] = csr_off, csr_ids[:ne.value]
        if b_off is not None:
            res["barle_off"], res["barle"] = b_off, b_bytes[:nb.value]
        res["shadow"] = shadow
        return res

    def trace_range(self, v0: int, v1: int, csr: bool = True, barle: bool = False) -> dict:
        """The last Stage 1 result for voxels [v0, v1) only: offsets rebased
        to 0, the lists and the shadow words (for scenes whose full lists are
        too large to copy to the host)."""
        L = lib()
        n = v1 - v0
        w = C.c_int()
        _check(L.solar_gpu_trace_sizes(self.h, None, None, C.byref(w), None, None))
        res = {"shadow": np.zeros((n, w.value), np.uint32)}
        co = np.zeros(n + 1, np.int64) if csr else None
        bo = np.zeros(n + 1, np.int64) if barle else None
        _check(L.solar_gpu_trace_copy_range(self.h, v0, v1, _p(co), None, _p(bo), None, _p(res["shadow"])))
        ids = np.zeros(max(1, int(co[-1] - co[0])), np.int32) if csr else None
        byt = np.zeros(max(1, int(bo[-1] - bo[0])), np.uint8) if barle else None
        _check(L.solar_gpu_trace_copy_range(self.h, v0, v1, None, _p(ids), None, _p(byt), None))
        if csr:
            res["csr_off"], res["csr_ids"] = co - co[0], ids[:int(co[-1] - co[0])]
        if barle:
            res["barle_off"], res["barle"] = bo - bo[0], byt[:int(bo[-1] - bo[0])]
        return res

    def timings(self) -> list[float]:
        """[setup, stage 1, stage 2/3, total] of the last run, ms (CUDA events)."""
        ms = (C.c_double * 4)()
        n = lib().solar_gpu_last_timings(self.h, ms, 4)
        if n < 0:
            _check(n)
        return list(ms)[:n]

    KERNEL_GROUPS = ("setup", "trace", "dedupe", "csr", "barle", "solar", "reflect", "finalize", "group")

    def kernel_times(self) -> dict:
        """{group: (ms, launches)} of the last run made with time_kernels=1."""
        ms = (C.c_double * 9)()
        ln = (C.c_longlong * 9)()
        n = lib().solar_gpu_kernel_times(self.h, ms, ln, 9)
        if n < 0:
            _check(n)
        return {g: (ms[i], int(ln[i])) for i, g in enumerate(self.KERNEL_GROUPS[:n])}

    def reflection_entries(self) -> int:
        """Weighted/union entries streamed per hour block in the last run."""
        return int(lib().solar_gpu_last_reflection_entries(self.h))

    def staged_rows(self) -> int:
        """Slab rows the tile kernel staged per hour block in the last run."""
        return int(lib().solar_gpu_last_staged_rows(self.h))

    def weighted_entries(self) -> int:
        """Nonzero reflection weights of the last run (one FMA per hour each)."""
        return int(lib().solar_gpu_last_weighted_entries(self.h))

    def launches(self) -> int:
        return int(lib().solar_gpu_last_launch_count(self.h))
