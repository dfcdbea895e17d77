"""Caller-side input preparation for the annual irradiance path.

This module plays the role of the reference CLI (``src/main.cpp:87-127``): it
produces, in host memory, every array the two drop-in entry points take.  It
is not part of the GPU hot path.  It contains

* a seeded synthetic DSM generator (value-noise ground, rectangular flat-roof
  buildings, Gaussian tree bumps) and a seeded synthetic TMY series;
* the hourly PSA sun position series (``include/sun_position.h:24-108``),
  evaluated with the same double-precision formula and rounded to float;
* the column-drop wall voxelization and top slope/aspect
  (``src/voxelization.cpp:10-97``) and the voxel array packing of
  ``src/main.cpp:112-127`` (top voxels in raster order, walls after, wall
  slope = pi/2).

Transcendentals are evaluated in double precision and rounded to float32 so
the arrays do not depend on the SIMD paths numpy picks on a given CPU.
"""
from __future__ import annotations

import calendar
import dataclasses
import datetime as _dt
import math

import numpy as np

HOURS_PER_YEAR = 8760  # include/pipeline_constants.h:10


# --------------------------------------------------------------------------
# Named workloads
# --------------------------------------------------------------------------

@dataclasses.dataclass(frozen=True)
class DsmConfig:
    """Parameters of one seeded synthetic DSM + site + TMY series."""
    name: str
    size: int                 # square grid side, cells of 1 m
    n_buildings: int
    n_trees: int
    roof_min: float = 4.0     # building height above local ground, m
    roof_max: float = 30.0
    side_min: int = 8
    side_max: int = 30
    tree_peak_min: float = 5.0
    tree_peak_max: float = 15.0
    tree_sigma: float = 2.0
    ground_amp: float = 3.0   # value-noise ground amplitude, m
    ground_cell: int = 16     # value-noise lattice spacing, cells
    lat: float = 46.56
    lon: float = 15.65
    tz: int = 1
    seed: int = 1


# The small plain-method case: 64x64, 12 buildings, 20 trees.
SMALL_64 = DsmConfig("dsm64", 64, 12, 20, seed=64)
# The 1024x1024 city: ~150 buildings; the tree count is chosen so the
# voxelized DSM holds about 1.5 M voxels.
CITY_1024 = DsmConfig("dsm1024", 1024, 150, 4600, seed=1024)
# The 4096x4096 city: ~2400 buildings up to 60 m, dense tree cover.
CITY_4096 = DsmConfig("dsm4096", 4096, 2400, 130000, roof_max=60.0, seed=4096)
# Mid-size case used by parity tests that must finish in seconds on the CPU oracle.
TOWN_160 = DsmConfig("dsm160", 160, 20, 60, seed=160)
# 256x256 and 512x512 cuts of the 1024 city's densities (profiling runs that
# must stay small; at 512 the hour-block slab no longer fits in L2).
CITY_256 = DsmConfig("dsm256", 256, 10, 290, seed=256)
CITY_512 = DsmConfig("dsm512", 512, 38, 1150, seed=512)

CONFIGS = {c.name: c for c in (SMALL_64, TOWN_160, CITY_256, CITY_512, CITY_1024, CITY_4096)}


# --------------------------------------------------------------------------
# DSM
# --------------------------------------------------------------------------

def _value_noise(rng: np.random.Generator, n: int, cell: int, amp: float) -> np.ndarray:
    """Single-octave value noise: uniform lattice values, smoothstep-bilinear."""
    m = n // cell + 2
    lattice = rng.random((m, m))
    coord = np.arange(n, dtype=np.float64) / cell
    i0 = np.floor(coord).astype(np.int64)
    f = coord - i0
    s = f * f * (3.0 - 2.0 * f)
    a = lattice[np.ix_(i0, i0)]
    b = lattice[np.ix_(i0, i0 + 1)]
    c = lattice[np.ix_(i0 + 1, i0)]
    d = lattice[np.ix_(i0 + 1, i0 + 1)]
    sy = s[:, None]
    sx = s[None, :]
    top = a * (1 - sx) + b * sx
    bot = c * (1 - sx) + d * sx
    return (top * (1 - sy) + bot * sy) * amp


def make_dsm(cfg: DsmConfig) -> np.ndarray:
    """Seeded synthetic DSM, float32 [size, size], row-major (y, x)."""
    rng = np.random.default_rng(cfg.seed)
    n = cfg.size
    ground = _value_noise(rng, n, cfg.ground_cell, cfg.ground_amp)
    z = ground.copy()
    for _ in range(cfg.n_buildings):
        w = int(rng.integers(cfg.side_min, cfg.side_max + 1))
        h = int(rng.integers(cfg.side_min, cfg.side_max + 1))
        w = min(w, n)
        h = min(h, n)
        x0 = int(rng.integers(0, n - w + 1))
        y0 = int(rng.integers(0, n - h + 1))
        roof = ground[y0:y0 + h, x0:x0 + w].max() + rng.uniform(cfg.roof_min, cfg.roof_max)
        np.maximum(z[y0:y0 + h, x0:x0 + w], roof, out=z[y0:y0 + h, x0:x0 + w])
    r = int(math.ceil(4 * cfg.tree_sigma))
    off = np.arange(-r, r + 1)
    for _ in range(cfg.n_trees):
        cx = rng.uniform(0, n)
        cy = rng.uniform(0, n)
        peak = rng.uniform(cfg.tree_peak_min, cfg.tree_peak_max)
        ix = int(cx) + off
        iy = int(cy) + off
        ix = ix[(ix >= 0) & (ix < n)]
        iy = iy[(iy >= 0) & (iy < n)]
        if ix.size == 0 or iy.size == 0:
            continue
        dx = (ix + 0.5 - cx)[None, :]
        dy = (iy + 0.5 - cy)[:, None]
        bump = peak * np.exp(-(dx * dx + dy * dy) / (2.0 * cfg.tree_sigma ** 2))
        sub = z[np.ix_(iy, ix)]
        z[np.ix_(iy, ix)] = np.maximum(sub, ground[np.ix_(iy, ix)] + bump)
    return z.astype(np.float32)


# --------------------------------------------------------------------------
# Sun positions (PSA), include/sun_position.h:24-108
# --------------------------------------------------------------------------

def sun_positions(lon: float, lat: float, tz: int, year: int = 2026) -> np.ndarray:
    """Hourly (azimuth_deg, altitude_deg) float32 [8760, 2] for a non-leap year.

    Same formula and order as ``SunPositionCalculator::calc``: days 1..365 of
    ``year`` (month/day from the calendar), hours 0..23 local standard time
    shifted to UT by the fixed ``tz`` offset.  ``lon``/``lat`` are taken as
    float32 values, as the reference stores them.
    """
    lon = float(np.float32(lon))
    lat = float(np.float32(lat))
    n_days = 366 if calendar.isleap(year) else 365
    kpi = 3.14159265358979323846
    krad = kpi / 180.0
    two_pi = 2.0 * kpi
    out = np.empty((n_days * 24, 2), dtype=np.float32)
    k = 0
    jan1 = _dt.date(year, 1, 1)
    for doy in range(1, n_days + 1):
        date = jan1 + _dt.timedelta(days=doy - 1)
        month, day = date.month, date.day
        for hour in range(24):
            utc_hours = hour - tz + 0 / 60.0
            aux1 = int((month - 14) / 12)  # C integer division truncates toward zero
            aux2 = (_cdiv(1461 * (year + 4800 + aux1), 4)
                    + _cdiv(367 * (month - 2 - 12 * aux1), 12)
                    - _cdiv(3 * _cdiv(year + 4900 + aux1, 100), 4)
                    + day - 32075)
            jd = float(aux2) - 0.5 + utc_hours / 24.0 - 2451545.0
            omega = 2.1429 - 0.0010394594 * jd
            mean_lon = 4.8950630 + 0.017202791698 * jd
            anomaly = 6.2400600 + 0.0172019699 * jd
            ecl_lon = (mean_lon + 0.03341607 * math.sin(anomaly)
                       + 0.00034894 * math.sin(2 * anomaly) - 0.0001134
                       - 0.0000203 * math.sin(omega))
            ecl_obl = 0.4090928 - 6.2140e-9 * jd + 0.0000396 * math.cos(omega)
            sin_el = math.sin(ecl_lon)
            dy = math.cos(ecl_obl) * sin_el
            dx = math.cos(ecl_lon)
            ra = math.atan2(dy, dx)
            if ra < 0.0:
                ra += two_pi
            decl = math.asin(math.sin(ecl_obl) * sin_el)
            gmst = 6.6974243242 + 0.0657098283 * jd + utc_hours
            lmst = (gmst * 15.0 + lon) * krad
            ha = lmst - ra
            lat_r = lat * krad
            cos_lat = math.cos(lat_r)
            sin_lat = math.sin(lat_r)
            cos_ha = math.cos(ha)
            zen = math.acos(cos_lat * cos_ha * math.cos(decl) + math.sin(decl) * sin_lat)
            az_y = -math.sin(ha)
            az_x = math.tan(decl) * cos_lat - sin_lat * cos_ha
            az = math.atan2(az_y, az_x)
            if az < 0.0:
                az += two_pi
            az /= krad
            parallax = (6371.01 / 149597890.0) * math.sin(zen)
            zen = (zen + parallax) / krad
            out[k, 0] = np.float32(az)
            out[k, 1] = np.float32(90.0 - zen)
            k += 1
    return out[:HOURS_PER_YEAR]


def _cdiv(a: int, b: int) -> int:
    """C/C++ integer division (truncation toward zero)."""
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


# --------------------------------------------------------------------------
# Synthetic TMY
# --------------------------------------------------------------------------

def make_tmy(sun: np.ndarray, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Seeded synthetic hourly DNI / DHI, float32 [8760] each (W/m^2).

    DNI = 900 * exp(-0.15 * AM) * c_t, with AM the Kasten-Young air mass of
    the hour's sun altitude (0 when the sun is below the horizon) and c_t an
    AR(1) cloud factor x_t = 0.8 x_{t-1} + e_t, e_t ~ N(0, 0.25^2),
    c_t = clip(0.75 + x_t, 0, 1).  DHI = f * GHI with f ~ U(0.1, 0.5) drawn
    once per day and GHI = DNI cos z + DHI, i.e. DHI = f/(1-f) * DNI cos z.
    """
    rng = np.random.default_rng(seed)
    alt = sun[:, 1].astype(np.float64)
    dni = np.zeros(HOURS_PER_YEAR)
    dhi = np.zeros(HOURS_PER_YEAR)
    f_day = rng.uniform(0.1, 0.5, size=365)
    eps = rng.normal(0.0, 0.25, size=HOURS_PER_YEAR)
    x = 0.0
    for t in range(HOURS_PER_YEAR):
        x = 0.8 * x + eps[t]
        c = min(1.0, max(0.0, 0.75 + x))
        a = alt[t]
        if a <= 0.0:
            continue
        zdeg = 90.0 - a
        cz = math.cos(math.radians(zdeg))
        am = 1.0 / (cz + 0.50572 * (96.07995 - zdeg) ** -1.6364)
        dni[t] = 900.0 * math.exp(-0.15 * am) * c
        f = f_day[t // 24]
        dhi[t] = f / (1.0 - f) * dni[t] * cz
    return dni.astype(np.float32), dhi.astype(np.float32)


# --------------------------------------------------------------------------
# Voxelization, src/voxelization.cpp:10-97 and src/main.cpp:112-127
# --------------------------------------------------------------------------

_OPEN_OUTSIDE = np.float32(-1e30)
_TWO_PI_F = np.float32(2.0) * np.float32(math.pi)


def _atan2_f32(y: np.ndarray, x: np.ndarray) -> np.ndarray:
    return np.arctan2(y.astype(np.float64), x.astype(np.float64)).astype(np.float32)


def detect_wall_voxels(heights: np.ndarray, voxel_size: float = 1.0):
    """Column-drop wall voxels: (parent_idx int32, z float32, aspect float32).

    Walls are ordered by parent pixel in raster order, then from the top of
    the drop downwards, as ``detect_wall_voxels`` appends them.
    """
    h = heights.astype(np.float32)
    H, W = h.shape
    vs = np.float32(voxel_size)
    pad = np.full((H + 2, W + 2), _OPEN_OUTSIDE, dtype=np.float32)
    pad[1:-1, 1:-1] = h
    hE = pad[1:-1, 2:]
    hW = pad[1:-1, :-2]
    hN = pad[:-2, 1:-1]
    hS = pad[2:, 1:-1]
    half = _OPEN_OUTSIDE * np.float32(0.5)
    cE = np.where(hE <= half, h, hE)
    cW = np.where(hW <= half, h, hW)
    cN = np.where(hN <= half, h, hN)
    cS = np.where(hS <= half, h, hS)
    mn = np.minimum(np.minimum(cE, cW), np.minimum(cN, cS))
    drop = (h - mn).astype(np.float32)
    has = drop > vs
    nvox = np.where(has, (drop / vs).astype(np.float32), np.float32(0)).astype(np.int64)
    nvox[~has] = 0
    flat = nvox.ravel()
    parents = np.repeat(np.arange(H * W, dtype=np.int64), flat)
    if parents.size == 0:
        return (np.zeros(0, np.int32), np.zeros(0, np.float32), np.zeros(0, np.float32))
    starts = np.cumsum(flat) - flat
    v = np.arange(parents.size, dtype=np.int64) - np.repeat(starts, flat)
    z0 = h.ravel()[parents]
    zz = (z0 - (v.astype(np.float32) + np.float32(0.5)) * vs).astype(np.float32)
    zero = np.float32(0.0)
    oE = np.maximum(zero, zz - hE.ravel()[parents])
    oW = np.maximum(zero, zz - hW.ravel()[parents])
    oN = np.maximum(zero, zz - hN.ravel()[parents])
    oS = np.maximum(zero, zz - hS.ravel()[parents])
    vx = (oE - oW).astype(np.float32)
    vy = (oN - oS).astype(np.float32)
    asp = _atan2_f32(vx, vy)
    asp = np.where(asp < 0, (asp + _TWO_PI_F).astype(np.float32), asp).astype(np.float32)
    return parents.astype(np.int32), zz, asp


def top_slope_aspect(heights: np.ndarray, scale: float = 1.0):
    """Central-difference slope/aspect per top pixel (radians, float32)."""
    h = heights.astype(np.float32)
    H, W = h.shape
    gx = np.arange(W)
    gy = np.arange(H)
    gxL = np.maximum(gx - 1, 0)
    gxR = np.minimum(gx + 1, W - 1)
    gyU = np.maximum(gy - 1, 0)
    gyD = np.minimum(gy + 1, H - 1)
    zL = h[:, gxL]
    zR = h[:, gxR]
    zU = h[gyU, :]
    zD = h[gyD, :]
    sc = np.float32(scale)
    dxden = ((gxR - gxL).astype(np.float32) * sc)[None, :]
    dyden = ((gyD - gyU).astype(np.float32) * sc)[:, None]
    dx = ((zR - zL) / dxden).astype(np.float32)
    dy = ((zD - zU) / dyden).astype(np.float32)
    mag = np.sqrt((dx * dx + dy * dy).astype(np.float32)).astype(np.float32)
    slope = _atan2_f32(mag, np.ones_like(mag))
    asp = _atan2_f32(-dx, dy)
    asp = np.where(asp < 0, (asp + _TWO_PI_F).astype(np.float32), asp).astype(np.float32)
    return slope.ravel(), asp.ravel()


# --------------------------------------------------------------------------
# One full set of API inputs
# --------------------------------------------------------------------------

@dataclasses.dataclass
class Scene:
    """Every host array the two drop-in entry points take."""
    name: str
    grid: np.ndarray          # float32 [H*W] raster order
    width: int
    height: int
    num_total: int
    num_top: int
    pixel_parent: np.ndarray  # int32 [num_total]
    wall_z: np.ndarray        # float32 [num_total - num_top]
    max_height: float
    sun: np.ndarray           # float32 [8760, 2] (azimuth_deg, altitude_deg)
    direct: np.ndarray        # float32 [8760]
    diffuse: np.ndarray       # float32 [8760]
    slopes: np.ndarray        # float32 [num_total]
    aspects: np.ndarray       # float32 [num_total]

    def arrays(self) -> dict:
        return {k: getattr(self, k) for k in (
            "grid", "pixel_parent", "wall_z", "sun", "direct", "diffuse", "slopes", "aspects")}


def voxelize(heights: np.ndarray, voxel_size: float = 1.0):
    """Voxel arrays packed as ``src/main.cpp:112-127`` packs them."""
    H, W = heights.shape
    num_top = H * W
    parents, wz, wasp = detect_wall_voxels(heights, voxel_size)
    slope_t, asp_t = top_slope_aspect(heights, voxel_size)
    num_total = num_top + parents.size
    pixel_parent = np.concatenate([np.arange(num_top, dtype=np.int32), parents])
    slopes = np.concatenate([slope_t, np.full(parents.size, np.float32(math.pi) * np.float32(0.5),
                                              dtype=np.float32)])
    aspects = np.concatenate([asp_t, wasp]).astype(np.float32)
    return num_total, num_top, pixel_parent, wz.astype(np.float32), slopes.astype(np.float32), aspects


def make_scene(cfg: DsmConfig | str, heights: np.ndarray | None = None) -> Scene:
    """Builds the full seeded input set for one named workload."""
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    z = make_dsm(cfg) if heights is None else heights.astype(np.float32)
    H, W = z.shape
    num_total, num_top, pp, wz, sl, asp = voxelize(z, 1.0)
    sun = sun_positions(cfg.lon, cfg.lat, cfg.tz)
    dni, dhi = make_tmy(sun, cfg.seed + 7)
    return Scene(cfg.name, z.ravel().copy(), W, H, num_total, num_top, pp, wz,
                 float(z.max()), sun, dni, dhi, sl, asp)


def scene_from_heightmap(name: str, heights: np.ndarray, voxel_size: float, lon: float, lat: float, tz: int,
                         direct: np.ndarray | None = None, diffuse: np.ndarray | None = None, seed: int = 1) -> Scene:
    """The inputs the reference CLI builds from a heightmap (src/main.cpp:70-127):
    voxelization with the raster's pixel size, the sun series of the site,
    and the given hourly TMY series (the seeded synthetic series when none
    are given)."""
    z = np.asarray(heights, np.float32)
    H, W = z.shape
    num_total, num_top, pp, wz, sl, asp = voxelize(z, voxel_size)
    sun = sun_positions(lon, lat, tz)
    if direct is None or diffuse is None:
        direct, diffuse = make_tmy(sun, seed + 7)
    return Scene(name, z.ravel().copy(), W, H, num_total, num_top, pp, wz, float(z.max()), sun,
                 np.asarray(direct, np.float32)[:8760], np.asarray(diffuse, np.float32)[:8760], sl, asp)


def scene_from_arrays(name: str, d: dict, width: int, height: int) -> Scene:
    """Rebuilds a Scene from stored arrays (golden fixtures)."""
    grid = np.asarray(d["grid"], np.float32)
    pp = np.asarray(d["pixel_parent"], np.int32)
    num_top = width * height
    return Scene(name, grid, width, height, int(pp.size), num_top, pp,
                 np.asarray(d["wall_z"], np.float32), float(grid.max()),
                 np.asarray(d["sun"], np.float32), np.asarray(d["direct"], np.float32),
                 np.asarray(d["diffuse"], np.float32), np.asarray(d["slopes"], np.float32),
                 np.asarray(d["aspects"], np.float32))
