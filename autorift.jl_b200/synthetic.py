"""Seeded synthetic image pairs with the shapes and statistics of the benchmark workloads.

No imagery is shipped or downloaded: every workload is generated from a seed. The generators
follow the workload descriptions (noise texture, Gaussian filtering, known displacement
fields) and the reference's own test helpers (`synthetic_texture`, `shifted_pair`,
test/utils.jl:164-321) in spirit; numpy's PCG64 stands in for Julia's MersenneTwister, so the
images are not bit-identical to the reference's tests.
"""

from __future__ import annotations

import numpy as np

try:  # scipy is used for Gaussian filtering, Fourier shifts and bicubic warps
    from scipy import ndimage as _ndi
except Exception:  # pragma: no cover - scipy is part of the image
    _ndi = None


def synthetic_texture(shape, seed: int = 0, dtype=np.float32) -> np.ndarray:
    """Band-limited noise in [0, 1]: three 3x3 box blurs of white noise."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    for _ in range(3):
        a = _box3(a)
    a -= a.min()
    m = a.max()
    if m > 0:
        a /= m
    if np.issubdtype(np.dtype(dtype), np.integer):
        return np.round(a * np.iinfo(dtype).max).astype(dtype)
    return a.astype(dtype)


def _box3(a: np.ndarray) -> np.ndarray:
    """Mean over the in-bounds 3x3 neighbourhood."""
    p = np.pad(a, 1)
    c = np.pad(np.ones_like(a), 1)
    s = sum(p[1 + di:1 + di + a.shape[0], 1 + dj:1 + dj + a.shape[1]]
            for di in (-1, 0, 1) for dj in (-1, 0, 1))
    n = sum(c[1 + di:1 + di + a.shape[0], 1 + dj:1 + dj + a.shape[1]]
            for di in (-1, 0, 1) for dj in (-1, 0, 1))
    return s / n


def shift_bilinear(a: np.ndarray, dx: float, dy: float) -> np.ndarray:
    """`a` translated by (+dx, +dy): samples a at (i - dy, j - dx), clamped at the border."""
    nr, nc = a.shape
    ii, jj = np.meshgrid(np.arange(nr, dtype=np.float64), np.arange(nc, dtype=np.float64),
                         indexing="ij")
    y = ii - dy
    x = jj - dx
    i0 = np.floor(y).astype(np.int64)
    j0 = np.floor(x).astype(np.int64)
    fy = y - i0
    fx = x - j0
    out = np.zeros_like(a, dtype=np.float64)
    for di, wi in ((0, 1 - fy), (1, fy)):
        for dj, wj in ((0, 1 - fx), (1, fx)):
            out += wi * wj * a[np.clip(i0 + di, 0, nr - 1), np.clip(j0 + dj, 0, nc - 1)]
    return out


def rotate_bilinear(a: np.ndarray, deg: float) -> np.ndarray:
    """`a` rotated by `deg` degrees about its centre ((nr + 1) / 2, (nc + 1) / 2, 1-based):
    each output pixel samples `a` by the inverse rotation, bilinearly, and is zero where a
    neighbour falls outside `a`. A scene rotation for the rotation-search workloads, in the
    convention of the reference's `rotate_bilinear` test helper (test/utils.jl:208-224)."""
    nr, nc = a.shape
    ii, jj = np.meshgrid(np.arange(1, nr + 1, dtype=np.float64),
                         np.arange(1, nc + 1, dtype=np.float64), indexing="ij")
    yc, xc = (nr + 1) / 2, (nc + 1) / 2
    r = np.deg2rad(deg)
    s, c = np.sin(r), np.cos(r)
    dy, dx = ii - yc, jj - xc
    y = yc + c * dy + s * dx - 1
    x = xc - s * dy + c * dx - 1
    i0 = np.floor(y).astype(np.int64)
    j0 = np.floor(x).astype(np.int64)
    fy = y - i0
    fx = x - j0
    out = np.zeros_like(a, dtype=np.float64)
    for di, wi in ((0, 1 - fy), (1, fy)):
        for dj, wj in ((0, 1 - fx), (1, fx)):
            out += wi * wj * a[np.clip(i0 + di, 0, nr - 1), np.clip(j0 + dj, 0, nc - 1)]
    out[(i0 < 0) | (j0 < 0) | (i0 + 1 > nr - 1) | (j0 + 1 > nc - 1)] = 0.0
    return out.astype(a.dtype) if a.dtype.kind == "f" else out


def shifted_pair(n: int, shift, seed: int = 0, dtype=np.float32):
    """(reference, secondary) where secondary is reference displaced by shift = (dx, dy)."""
    dx, dy = shift
    pad = int(np.ceil(max(abs(dx), abs(dy)))) + 2
    big = synthetic_texture((n + 2 * pad, n + 2 * pad), seed=seed, dtype=np.float64)
    ref = big[pad:pad + n, pad:pad + n]
    sec = shift_bilinear(big, dx, dy)[pad:pad + n, pad:pad + n]
    if np.issubdtype(np.dtype(dtype), np.integer):
        mx = np.iinfo(dtype).max
        conv = lambda v: np.round(np.clip(v, 0, 1) * mx).astype(dtype)
    else:
        conv = lambda v: v.astype(dtype)
    return conv(ref), conv(sec)


# ---------------------------------------------------------------------------------------------
# Benchmark workloads


def plain_512_pair(seed: int = 1, dx: float = 3.37, dy: float = -1.82):
    """512x512 Float32 pair: filtered noise (sigma 1.5, mean 0.5, std 0.1) and its Fourier shift
    by (dx, dy) plus N(0, 0.01) noise. Returns (image1, image2, (dx, dy))."""
    rng = np.random.default_rng(seed)
    a = _ndi.gaussian_filter(rng.standard_normal((512, 512)), 1.5)
    a = (a - a.mean()) / a.std() * 0.1 + 0.5
    spec = _ndi.fourier_shift(np.fft.fft2(a), (dy, dx))
    b = np.real(np.fft.ifft2(spec))
    b = b + np.random.default_rng(seed + 1).normal(0.0, 0.01, b.shape)
    return a.astype(np.float32), b.astype(np.float32), (dx, dy)


def plain_512_points(spacing: int = 16, margin: int = 32, n: int = 512, chip: int = 32,
                     radius: int = 25):
    """Centres every 16 px with a 32 px margin (29 x 29 = 841), 1-based coordinates."""
    from .points import gridpoints_xy
    c = np.arange(margin, n - margin + 1, spacing, dtype=np.float64)
    return gridpoints_xy(c, c, chip_size=chip, search_radius=radius)


def gaussian_bumps(shape, n_bumps: int, max_amp: float, widths=(300.0, 800.0), border: int = 200,
                   seed: int = 7):
    """Smooth displacement field (dx, dy): a sum of Gaussian bumps, zero within `border` px of
    the edge (tapered), peak amplitude up to `max_amp`."""
    rng = np.random.default_rng(seed)
    nr, nc = shape
    border = min(border, int(0.2 * min(nr, nc)))  # small scenes keep a proportional border
    yy = np.arange(nr, dtype=np.float64)[:, None]
    xx = np.arange(nc, dtype=np.float64)[None, :]
    fx = np.zeros(shape)
    fy = np.zeros(shape)
    for _ in range(n_bumps):
        cy = rng.uniform(border + 0.15 * nr, nr - border - 0.15 * nr)
        cx = rng.uniform(border + 0.15 * nc, nc - border - 0.15 * nc)
        w = rng.uniform(*widths) / 2.0
        amp = rng.uniform(0.3, 1.0) * max_amp
        ang = rng.uniform(0, 2 * np.pi)
        g = np.exp(-(((yy - cy) ** 2) + ((xx - cx) ** 2)) / (2 * w * w))
        fx += amp * np.cos(ang) * g
        fy += amp * np.sin(ang) * g
    # Taper to zero motion over the border.
    ty = np.clip(np.minimum(yy, nr - 1 - yy) / border, 0, 1)
    tx = np.clip(np.minimum(xx, nc - 1 - xx) / border, 0, 1)
    taper = np.minimum(ty, tx)
    taper = taper * taper * (3 - 2 * taper)
    m = max(np.abs(fx).max(), np.abs(fy).max(), 1e-12)
    scale = max_amp / m
    return fx * taper * scale, fy * taper * scale


def scale_u16_pair(n: int = 4096, seed: int = 11, max_amp: float = 15.0, noise: float = 0.02,
                   nodata: float = 0.03, sigma: float = 2.0, mean: float = 8000.0,
                   std: float = 1500.0, dtype=np.uint16):
    """UInt16 pair at scale: filtered noise (sigma 2) mapped to mean 8000, std 1500, clipped;
    the secondary is a bicubic warp by a 6-bump field plus 2% Gaussian noise (of the image
    std) and 3% zero-valued no-data blobs of radius 20-80 px. `mean`, `std` and `dtype`
    produce the same scene at another bit depth.

    Returns (image1, image2, secondary_valid, (fx, fy)) with (fx, fy) the imposed feature
    motion in pixels (the tracker reports its negative)."""
    hi = float(np.iinfo(dtype).max)
    rng = np.random.default_rng(seed)
    a = _ndi.gaussian_filter(rng.standard_normal((n, n)).astype(np.float32), sigma)
    a = (a - a.mean()) / a.std() * std + mean
    a = np.clip(a, 0, hi)
    fx, fy = gaussian_bumps((n, n), 6, max_amp, seed=seed + 1)
    yy, xx = np.meshgrid(np.arange(n, dtype=np.float32), np.arange(n, dtype=np.float32),
                         indexing="ij")
    coords = np.stack([yy - fy.astype(np.float32), xx - fx.astype(np.float32)])
    del yy, xx
    b = _ndi.map_coordinates(a, coords, order=3, mode="nearest")
    del coords
    b = b + rng.normal(0.0, noise * std, b.shape).astype(np.float32)
    b = np.clip(np.round(b), 0, hi).astype(dtype)
    img1 = np.round(a).astype(dtype)
    # No-data blobs.
    holes = np.zeros((n, n), bool)
    target = nodata * n * n
    covered = 0
    while covered < target:
        r = rng.uniform(20, 80)
        cy, cx = rng.uniform(0, n, 2)
        y0, y1 = int(max(cy - r, 0)), int(min(cy + r + 1, n))
        x0, x1 = int(max(cx - r, 0)), int(min(cx + r + 1, n))
        yy, xx = np.ogrid[y0:y1, x0:x1]
        disk = (yy - cy) ** 2 + (xx - cx) ** 2 <= r * r
        new = disk & ~holes[y0:y1, x0:x1]
        holes[y0:y1, x0:x1] |= disk
        covered += int(new.sum())
    b[holes] = 0
    return img1, b, ~holes, (fx, fy)


def batching_points(n: int, fx_down, fy_down, seed: int = 3, spacing: int = 8, margin: int = 24):
    """The batching configuration's point set on an n x n scene: fractional centres on a
    `spacing` px lattice with +-0.5 px jitter, per-point search radii uniform in [4, 48], and
    integer priors from the 4x-downsampled imposed feature motion (`fx_down`, `fy_down` =
    f[::4, ::4]) rounded, plus a uniform error of up to 3 px (the tracker reports the negative of
    the motion). Returns the PointSet fields x, y, radius, dx_prior, dy_prior as (m, m) arrays
    in Julia's layout."""
    rng = np.random.default_rng(seed)
    c = np.arange(margin, n - margin, spacing, dtype=np.float64)
    X, Y = np.meshgrid(c, c)  # rows follow y
    X = np.asfortranarray(X + rng.uniform(-0.5, 0.5, X.shape))
    Y = np.asfortranarray(Y + rng.uniform(-0.5, 0.5, Y.shape))
    r = rng.integers(4, 49, X.shape)
    iy = np.clip(np.round(Y - 1).astype(int) // 4, 0, fx_down.shape[0] - 1)
    ix = np.clip(np.round(X - 1).astype(int) // 4, 0, fx_down.shape[1] - 1)
    dx0 = np.round(-fx_down[iy, ix]) + rng.integers(-3, 4, X.shape)
    dy0 = np.round(-fy_down[iy, ix]) + rng.integers(-3, 4, X.shape)
    return X, Y, r, dx0, dy0
