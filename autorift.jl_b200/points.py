"""Search points (src/points.jl).

`PointSet` holds the reference's eight SoA fields. Arrays are indexed like Julia's
(`[row, col]` for a gridded set) and flattened in Julia's memory order (column-major) when they
cross the C ABI, so a gridded point set round-trips to a gridded result.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, replace

import numpy as np

FIELDS = ("x", "y", "radius_x", "radius_y", "dx_prior", "dy_prior", "chip_size_x",
          "chip_size_y")
_FLOAT_FIELDS = ("x", "y", "dx_prior", "dy_prior")


@dataclass
class PointSet:
    """Where to correlate and with what geometry (src/points.jl:50-74)."""

    x: np.ndarray
    y: np.ndarray
    radius_x: np.ndarray
    radius_y: np.ndarray
    dx_prior: np.ndarray
    dy_prior: np.ndarray
    chip_size_x: np.ndarray
    chip_size_y: np.ndarray

    def __post_init__(self):
        shape = np.shape(self.x)
        for name in FIELDS:
            a = np.asarray(getattr(self, name),
                           dtype=np.float64 if name in _FLOAT_FIELDS else np.int64)
            if a.shape != shape:
                raise ValueError(f"PointSet field `{name}` has shape {a.shape}, expected {shape} "
                                 "to match `x`")
            setattr(self, name, a)

    @property
    def shape(self):
        return self.x.shape

    @property
    def ndim(self):
        return self.x.ndim

    def __len__(self):
        return int(self.x.size)

    def flat(self, name: str) -> np.ndarray:
        """Field `name` flattened in Julia's memory order (`vec`, src/points.jl:276-281)."""
        return np.ascontiguousarray(getattr(self, name).ravel(order="F"))

    def __getitem__(self, idx):
        """Decimate or crop a gridded set, copying every field (src/points.jl:293-297)."""
        return PointSet(**{n: np.array(getattr(self, n)[idx]) for n in FIELDS})

    def copy(self):
        return PointSet(**{n: getattr(self, n).copy() for n in FIELDS})


def npoints(pts: PointSet) -> int:
    return len(pts)


def issearchable(pts: PointSet) -> np.ndarray:
    """Both radii positive (src/points.jl:116-117)."""
    return (pts.radius_x > 0) & (pts.radius_y > 0)


def nsearchable(pts: PointSet) -> int:
    return int(np.count_nonzero(issearchable(pts)))


def rebuild(pts: PointSet, **kw) -> PointSet:
    """A copy with the named fields replaced (src/points.jl:309-313)."""
    return replace(pts, **kw)


def _tofield(dtype, v, like: np.ndarray, name: str) -> np.ndarray:
    if np.isscalar(v):
        if dtype is np.int64 and float(v) != int(v):
            raise ValueError(f"expected an integer value, got {v}")
        return np.full(like.shape, v, dtype=dtype)
    a = np.asarray(v)
    if a.shape != like.shape:
        raise ValueError(f"`{name}` has shape {a.shape} but there are {like.shape} points")
    if dtype is np.int64:
        if np.any(a != np.round(a)):
            raise ValueError(f"expected an integer value in `{name}`")
        return a.astype(np.int64)
    return a.astype(np.float64)


def pointset(x, y, *, search_radius=25, search_radius_x=None, search_radius_y=None,
             chip_size=32, chip_size_x=None, chip_size_y=None, chip_aspect=1.0, dx_prior=0.0,
             dy_prior=0.0) -> PointSet:
    """Build a PointSet from centre coordinates (src/points.jl:149-182)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if x.shape != y.shape:
        raise ValueError(f"`x` and `y` must have the same shape, got {x.shape} and {y.shape}")
    if isinstance(search_radius, tuple):
        rx0, ry0 = search_radius
    else:
        rx0 = ry0 = search_radius
    rx = _tofield(np.int64, rx0 if search_radius_x is None else search_radius_x, x,
                  "search_radius_x")
    ry = _tofield(np.int64, ry0 if search_radius_y is None else search_radius_y, x,
                  "search_radius_y")
    csx = _tofield(np.int64, chip_size if chip_size_x is None else chip_size_x, x, "chip_size_x")
    if chip_size_y is None:
        # 2 * round(Int, c * chip_aspect / 2): Julia rounds half to even, as numpy does.
        csy = (2 * np.round(csx * float(chip_aspect) / 2)).astype(np.int64)
    else:
        csy = _tofield(np.int64, chip_size_y, x, "chip_size_y")
    dx = _tofield(np.float64, dx_prior, x, "dx_prior")
    dy = _tofield(np.float64, dy_prior, x, "dy_prior")
    return PointSet(x.copy(), y.copy(), rx, ry, dx, dy, csx, csy)


def gridpoints(imagesize, spacing: int, *, chip_size=32, chip_aspect=1.0, search_radius=25,
               search_radius_x=None, search_radius_y=None, **kw) -> PointSet:
    """A gridded PointSet inset so every chip and window fits (src/points.jl:231-265)."""
    if spacing <= 0:
        raise ValueError(f"`spacing` must be positive, got {spacing}")
    if isinstance(search_radius, tuple):
        rx0, ry0 = search_radius
    else:
        rx0 = ry0 = search_radius
    rx = rx0 if search_radius_x is None else search_radius_x
    ry = ry0 if search_radius_y is None else search_radius_y
    csx = int(np.max(chip_size))
    csy = 2 * int(round(csx * chip_aspect / 2))
    margin_x = -(-csx // 2) + int(np.max(rx)) + 1
    margin_y = -(-csy // 2) + int(np.max(ry)) + 1
    nrows, ncols = imagesize
    xs = np.arange(margin_x + 1, ncols - margin_x + 1, spacing, dtype=np.float64)
    ys = np.arange(margin_y + 1, nrows - margin_y + 1, spacing, dtype=np.float64)
    if xs.size == 0 or ys.size == 0:
        raise ValueError(
            f"no search center fits in a {nrows}x{ncols} image with chip {csx}x{csy} and search "
            f"radius {rx}x{ry}: a margin of {margin_y}x{margin_x} pixels is needed on each side. "
            "Use a smaller chip size or search radius.")
    return gridpoints_xy(xs, ys, chip_size=chip_size, chip_aspect=chip_aspect,
                         search_radius=search_radius, search_radius_x=search_radius_x,
                         search_radius_y=search_radius_y, **kw)


def gridpoints_xy(xs, ys, **kw) -> PointSet:
    """The explicit-coordinate form of gridpoints (src/points.jl:260-265)."""
    xs = np.asarray(xs, dtype=np.float64)
    ys = np.asarray(ys, dtype=np.float64)
    X = np.asfortranarray(np.broadcast_to(xs[None, :], (ys.size, xs.size)))
    Y = np.asfortranarray(np.broadcast_to(ys[:, None], (ys.size, xs.size)))
    return pointset(X, Y, **kw)


def sanitize(pts: PointSet, min_radius: int) -> int:
    """Normalise radii in place; returns the number left searchable (src/points.jl:332-346)."""
    bad = (pts.radius_x <= 0) | (pts.radius_y <= 0)
    pts.radius_x[bad] = 0
    pts.radius_y[bad] = 0
    ok = ~bad
    pts.radius_x[ok] = np.maximum(pts.radius_x[ok], min_radius)
    pts.radius_y[ok] = np.maximum(pts.radius_y[ok], min_radius)
    return int(np.count_nonzero(ok))


def chip_bounds(pts: PointSet, i):
    """1-based inclusive (rows, cols) of the chip cut from the secondary (src/points.jl:358-366)."""
    hx = int(pts.chip_size_x.flat[i]) // 2
    hy = int(pts.chip_size_y.flat[i]) // 2
    cx = math.floor(pts.x.flat[i] - pts.dx_prior.flat[i])
    cy = math.floor(pts.y.flat[i] - pts.dy_prior.flat[i])
    return (cy - hy, cy + hy - 1), (cx - hx, cx + hx - 1)


def search_bounds(pts: PointSet, i):
    """1-based inclusive (rows, cols) of the window cut from the reference (src/points.jl:385-395)."""
    hx = int(pts.chip_size_x.flat[i]) // 2
    hy = int(pts.chip_size_y.flat[i]) // 2
    rx = int(pts.radius_x.flat[i])
    ry = int(pts.radius_y.flat[i])
    cx = math.floor(pts.x.flat[i])
    cy = math.floor(pts.y.flat[i])
    return (cy - hy - ry, cy + hy + ry - 2), (cx - hx - rx, cx + hx + rx - 2)


def inbounds(pts: PointSet, i, imagesize) -> bool:
    """Whether point i's search window lies inside the image (src/points.jl:421-425)."""
    (r0, r1), (c0, c1) = search_bounds(pts, i)
    return r0 >= 1 and r1 <= imagesize[0] and c0 >= 1 and c1 <= imagesize[1]


def surface_size(pts: PointSet, i):
    return 2 * int(pts.radius_y.flat[i]), 2 * int(pts.radius_x.flat[i])
