"""The geometry behind the tracer's early exit (solargpu_b200/csrc/cone.cu),
checked on the CPU.

An upper ray may end with no hit once its height passes the bound of a cell
it has reached, because that bound covers every cell the ray can still visit.
The tables take the bound from a cone K between two consecutive primitive
vectors a, b of the Farey set of order 8 (chosen per direction from the
floats dX, dY the DDA adds), widened by a window of unsigned offsets
[-(r + a + b), r] per axis, r = 1 + ceil(2 L (L + 1) 2^-24).  This test walks
the float32 DDA of viewshed_kernels.cu:27-58 for directions of the traced
set and checks the claim the tables rest on: every cell a ray visits after a
cell c lies in c + e + K for some offset e of the window."""
import numpy as np

from oracle import oracle as O

ORDER = 8


def farey(n):
    """Primitive (p, q), 0 <= p, q <= n, by angle from (1, 0) to (0, 1)."""
    import functools
    from math import gcd
    v = [(p, q) for p in range(n + 1) for q in range(n + 1) if (p or q) and gcd(p, q) == 1]
    return sorted(v, key=functools.cmp_to_key(lambda a, b: -1 if a[0] * b[1] - a[1] * b[0] > 0 else 1))


def cone_of(F, dX, dY):
    """The cone (F[k], F[k + 1]) holding (1/dX, 1/dY) ~ (dY, dX), as the host
    code assigns it (exact products of small integers and floats)."""
    for k in range(len(F) - 1):
        if F[k][0] * dX - F[k][1] * dY >= 0 and dY * F[k + 1][1] - dX * F[k + 1][0] >= 0:
            return F[k], F[k + 1]
    raise AssertionError("direction outside every cone")


def dda_cells(cx, cy, gx, gy, steps):
    """Cells the float32 DDA visits after its start cell (unsigned: both
    coordinates grow along the ray)."""
    f = np.float32
    cx, cy = f(cx), f(cy)
    ox, oy = f(gx) + cx * f(2.0), f(gy) + cy * f(2.0)
    ax, ay = max(abs(cx), f(1e-8)), max(abs(cy), f(1e-8))
    dX, dY = f(1.0) / ax, f(1.0) / ay
    ix, iy = int(np.floor(ox)), int(np.floor(oy))
    tx = ((f(ix) + f(1.0)) - ox if cx >= 0 else ox - f(ix)) / ax
    ty = ((f(iy) + f(1.0)) - oy if cy >= 0 else oy - f(iy)) / ay
    sx, sy = (1 if cx >= 0 else -1), (1 if cy >= 0 else -1)
    out = []
    for _ in range(steps):
        if tx < ty:
            ix += sx
            tx = f(tx + dX)
        else:
            iy += sy
            ty = f(ty + dY)
        out.append((ix * sx, iy * sy))
    return np.array(out, np.int64), float(dX), float(dY)


def window_radius(L):
    return 1 + int(np.ceil(2.0 * L * (L + 1.0) / 16777216.0))


def test_farey_cones_are_unimodular_and_cover_the_quadrant():
    F = farey(ORDER)
    assert F[0] == (1, 0) and F[-1] == (0, 1)
    for a, b in zip(F[:-1], F[1:]):
        assert a[0] * b[1] - a[1] * b[0] == 1


def test_later_cells_lie_in_the_widened_cone():
    bins = O.sky_bins(np.zeros((8760, 2), np.float32) + np.float32([180.0, 30.0]))
    dirs, _, upper = O.directions(bins)
    up = np.flatnonzero(upper)
    rng = np.random.default_rng(3)
    F = farey(ORDER)
    steps = 160
    r = window_radius(steps + 4)
    checked = 0
    for d in rng.choice(up, 48, replace=False):
        cells, dX, dY = dda_cells(dirs[d, 0], dirs[d, 1], int(rng.integers(0, 50)), int(rng.integers(0, 50)), steps)
        a, b = cone_of(F, dX, dY)
        ex = np.arange(-(r + a[0] + b[0]), r + 1)
        ey = np.arange(-(r + a[1] + b[1]), r + 1)
        E = np.stack(np.meshgrid(ex, ey, indexing="ij"), -1).reshape(-1, 2)
        for k in range(0, steps - 1, 7):
            later = cells[k:] - cells[k]                                  # offsets, c itself included
            q = later[:, None, :] - E[None, :, :]                        # later - e for every e
            in_k = ((a[0] * q[..., 1] - a[1] * q[..., 0]) >= 0) & ((q[..., 0] * b[1] - q[..., 1] * b[0]) >= 0)
            assert in_k.any(axis=1).all(), (d, k)
            checked += later.shape[0]
    assert checked > 40000


def test_a_window_without_the_widening_would_not_do():
    """The window is needed: with r = 0 and no a + b reach some later cell
    falls outside c + K (the cone from the cell's corner misses cells the
    ray's line passes through next to it)."""
    bins = O.sky_bins(np.zeros((8760, 2), np.float32) + np.float32([180.0, 30.0]))
    dirs, _, upper = O.directions(bins)
    F = farey(ORDER)
    missed = 0
    for d in np.flatnonzero(upper)[::7]:
        cells, dX, dY = dda_cells(dirs[d, 0], dirs[d, 1], 11, 17, 120)
        a, b = cone_of(F, dX, dY)
        for k in range(0, 119, 5):
            q = cells[k:] - cells[k]
            ok = ((a[0] * q[:, 1] - a[1] * q[:, 0]) >= 0) & ((q[:, 0] * b[1] - q[:, 1] * b[0]) >= 0)
            missed += int((~ok).sum())
    assert missed > 0
