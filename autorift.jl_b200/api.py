"""The public API (src/api.jl): `autorift`, the `init` / `reinit!` / `autorift!` cache
lifecycle, `correlate_multichip` and `MultichipResult` (src/multichip.jl:74-137), on the GPU.

Python spells Julia's `reinit!` and `autorift!` as `reinit_` and `autorift_`.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .methods import (GardnerFilter, NoOutlierFilter, Params, chip_sizes, params as make_params,
                      upsampling)
from .points import PointSet, gridpoints
from .track import (ImagePair, PreparedPair, _measure_code, points_struct, prepare,
                    prepare_options, rotation_angles)


@dataclass
class MultichipResult:
    """Displacement over the full grid from all chip-size levels (src/multichip.jl:74-80)."""

    dx: np.ndarray
    dy: np.ndarray
    correlation: np.ndarray
    chip_size: np.ndarray
    interpolated: np.ndarray

    @property
    def shape(self):
        return self.dx.shape

    def __len__(self):
        return int(self.dx.size)


def multichip_params(p: Params) -> "_lib.ArMultichipParams":
    """The `ar_multichip_params` of a parameter set."""
    o = p.outliers
    if isinstance(o, GardnerFilter):
        kind, w, it, fr, tol, mad = 1, o.window, o.iterations, o.min_agree_fraction, o.agree_tolerance, o.mad_scale
    elif isinstance(o, NoOutlierFilter):
        kind, w, it, fr, tol, mad = 0, 5, 3, 8 / 25, 0.2, 4.0
    else:
        raise ValueError(f"{type(o).__name__} has no GPU implementation")
    if len(p.similarity) > len(chip_sizes(p)):
        raise ValueError(f"`similarity` names {len(p.similarity)} measures but there are only "
                         f"{len(chip_sizes(p))} chip-size levels.")
    levels = [_measure_code(m) for m in p.similarity]  # measure_at (src/types.jl:893-894)
    prm = _lib.ArMultichipParams(
        p.chip_size_base, p.chip_size_min, p.chip_size_max, p.chip_aspect,
        p.min_search_radius, p.coarse_stride, p.coarse_buffer, p.min_coarse_valid_fraction,
        upsampling(p.subpixel), _measure_code(p.similarity[0]), kind, w, it, fr, tol, mad,
        p.fill_window)
    if len(levels) > 1:
        prm.level_measure_count = len(levels)
        for i, m in enumerate(levels):
            prm.level_measures[i] = m
    rot = rotation_angles(p)
    if rot is not None:
        prm.rotation_count = rot.size
        prm.rotation_angles = rot.ctypes.data
        prm._angles = rot  # the array the struct points at lives as long as the struct
    return prm


def correlate_multichip(pair, grid: PointSet, p: Params | None = None, ctx=None) -> MultichipResult:
    """Correlate `pair` over the gridded `grid` at every chip-size level, finest first
    (src/multichip.jl:106-137). `pair` is a prepared pair (ImagePair of the correlation
    element type, or a PreparedPair already on the device)."""
    p = p if p is not None else make_params()
    ctx = ctx or _lib.default_context()
    if grid.ndim != 2:
        raise ValueError("correlate_multichip needs a gridded PointSet{2}")
    gr, gc = grid.shape
    n = gr * gc
    out = [np.empty(n, np.float32) for _ in range(3)]
    cs = np.empty(n, np.uint16)
    it = np.empty(n, np.uint8)
    if n:
        dp = pair.device(ctx)
        st, keep = points_struct(grid)
        prm = multichip_params(p)
        ctx.check(ctx.lib.ar_multichip(ctx.handle, dp.handle, ctypes.byref(st), gr, gc,
                                       ctypes.byref(prm), out[0].ctypes.data, out[1].ctypes.data,
                                       out[2].ctypes.data, cs.ctypes.data, it.ctypes.data))
    shp = lambda a: a.reshape((gr, gc), order="F")
    return MultichipResult(shp(out[0]), shp(out[1]), shp(out[2]), shp(cs), shp(it).astype(bool))


def nmeasured(r) -> int:
    return int(np.count_nonzero(~np.isnan(r.dx)))


def build_grid(imagesize, p: Params) -> PointSet:
    """The grid when the caller gives none (src/api.jl:339-347)."""
    return gridpoints(imagesize, p.grid_spacing, chip_size=p.chip_size_max,
                      chip_aspect=p.chip_aspect, search_radius_x=p.search_radius_x,
                      search_radius_y=p.search_radius_y, dx_prior=p.dx_prior,
                      dy_prior=p.dy_prior)


class Cache:
    """Prepared state for correlating many pairs with one configuration (src/api.jl:30-44)."""

    def __init__(self, p: Params, raw: ImagePair, prepared: PreparedPair, grid: PointSet, ctx):
        self.params = p
        self.raw = raw
        self.prepared = prepared
        self.grid = grid
        self.result = None
        self.isfresh = True
        self.ctx = ctx


def init(reference, secondary, *, reference_valid=None, secondary_valid=None, ctx=None,
         **kw) -> Cache:
    """Prepare to correlate a pair: resolve parameters, filter and quantise on the device,
    build the grid (src/api.jl:66-76)."""
    p = make_params(**kw)
    ctx = ctx or _lib.default_context()
    raw = ImagePair(reference, secondary, reference_valid, secondary_valid)
    prepared = prepare(raw, p, ctx)
    grid = build_grid(raw.shape, p)
    return Cache(p, raw, prepared, grid, ctx)


def reinit_(cache: Cache, *, reference=None, secondary=None, reference_valid=None,
            secondary_valid=None) -> Cache:
    """Point the cache at a new pair of the same size (src/api.jl:104-134): an omitted image
    keeps its value, an omitted mask follows its image, sizes must match."""
    if reference is None and secondary is None and reference_valid is None and secondary_valid is None:
        return cache
    old = cache.raw
    ref = old.reference if reference is None else reference
    sec = old.secondary if secondary is None else secondary

    def maskfor(img):
        if img is old.reference:
            return old.given_reference_valid
        if img is old.secondary:
            return old.given_secondary_valid
        return None

    rv = maskfor(ref) if reference_valid is None else reference_valid
    sv = maskfor(sec) if secondary_valid is None else secondary_valid
    if np.shape(ref) != old.shape or np.shape(sec) != old.shape:
        raise ValueError(f"new images are {np.shape(ref)} and {np.shape(sec)} but the cache was "
                         f"built for {old.shape}; build a new cache with `init` for a different "
                         "image size.")
    cache.raw = ImagePair(ref, sec, rv, sv)
    cache.prepared = prepare(cache.raw, cache.params, cache.ctx)
    cache.isfresh = True
    cache.result = None
    return cache


def autorift_(cache: Cache) -> MultichipResult:
    """Correlate the cache's pair; idempotent until the next reinit_ (src/api.jl:165-170)."""
    if not cache.isfresh and cache.result is not None:
        return cache.result
    cache.result = correlate_multichip(cache.prepared, cache.grid, cache.params, cache.ctx)
    cache.isfresh = False
    return cache.result


def autorift(reference, secondary, grid: PointSet | None = None, *, reference_valid=None,
             secondary_valid=None, ctx=None, **kw):
    """Displacement between two co-registered images (src/api.jl:210-274).

    With no grid: the full multi-chip-size search over `grid_spacing` points. With a gridded
    PointSet: the same search over it. With a scattered PointSet: one scale via `track`.
    """
    if grid is None:
        return autorift_(init(reference, secondary, reference_valid=reference_valid,
                              secondary_valid=secondary_valid, ctx=ctx, **kw))
    from .track import track
    p = make_params(**kw)
    ctx = ctx or _lib.default_context()
    prepared = prepare(ImagePair(reference, secondary, reference_valid, secondary_valid), p, ctx)
    if grid.ndim == 2:
        return correlate_multichip(prepared, grid, p, ctx)
    return track(prepared, grid, p, ctx=ctx)


class Ticket:
    """A queued autorift() request (ar_submit). Holds the request's host arrays until it has
    completed; `wait` returns its MultichipResult."""

    def __init__(self, ctx, ticket: int, keep, outs, shape):
        self.ctx = ctx
        self.ticket = int(ticket)
        self._keep = keep
        self._outs = outs
        self._shape = shape
        self._status = None

    def done(self) -> bool:
        """True once the request has completed (ar_poll)."""
        if self._status is not None:
            return True
        flag = ctypes.c_int(0)
        rc = self.ctx.lib.ar_poll(self.ctx.handle, self.ticket, ctypes.byref(flag))
        if flag.value:
            self._status = rc
            return True
        self.ctx.check(rc)
        return False

    def wait(self, timeout: float | None = None) -> MultichipResult:
        """Block until the request completes (ar_wait) and return its result; raises
        TimeoutError if it has not completed within `timeout` seconds, ArError if it failed."""
        if self._status is None:
            ms = -1 if timeout is None else max(0, int(round(timeout * 1000)))
            rc = self.ctx.lib.ar_wait(self.ctx.handle, self.ticket, ms)
            if rc == _lib.AR_ERR_TIMEOUT:
                raise TimeoutError(f"request {self.ticket} has not completed in {timeout} s")
            self._status = rc
        if self._status != _lib.AR_OK:
            self.ctx.check(self._status)
        gr, gc = self._shape
        shp = lambda a: a.reshape((gr, gc), order="F")
        o = self._outs
        return MultichipResult(shp(o[0]), shp(o[1]), shp(o[2]), shp(o[3]), shp(o[4]).astype(bool))

    def times(self):
        """(queued_ms, run_ms) of a completed request."""
        q, r = ctypes.c_double(), ctypes.c_double()
        self.ctx.check(self.ctx.lib.ar_request_times(self.ctx.handle, self.ticket, ctypes.byref(q),
                                                     ctypes.byref(r)))
        return q.value, r.value

    def release(self):
        if self._keep is not None and self.done():
            self.ctx.lib.ar_release(self.ctx.handle, self.ticket)
            self._keep = None

    def __del__(self):
        try:
            if self._keep is not None:
                if not self.done():
                    self.ctx.lib.ar_wait(self.ctx.handle, self.ticket, -1)  # buffers in use
                self.ctx.lib.ar_release(self.ctx.handle, self.ticket)
        except Exception:
            pass


def submit(reference, secondary, grid: PointSet | None = None, *, reference_valid=None,
           secondary_valid=None, ctx=None, **kw) -> Ticket:
    """Queue `autorift(reference, secondary; kw...)` on the context's request loop (ar_submit)
    and return at once; requests submitted together run concurrently on the device."""
    from .track import DTYPES, _colmajor, _mask_bytes
    p = make_params(**kw)
    ctx = ctx or _lib.default_context()
    ref = np.asarray(reference)
    sec = np.asarray(secondary)
    if ref.shape != sec.shape or ref.ndim != 2:
        raise ValueError(f"reference is {ref.shape} but secondary is {sec.shape}")
    if sec.dtype != ref.dtype:
        sec = sec.astype(ref.dtype)
    if ref.dtype not in DTYPES:
        raise TypeError(f"element type {ref.dtype} is not supported by the GPU correlator")
    grid = grid if grid is not None else build_grid(ref.shape, p)
    if grid.ndim != 2:
        raise ValueError("a request needs a gridded PointSet{2}")
    gr, gc = grid.shape
    n = gr * gc
    arrays = [_colmajor(ref), _colmajor(sec)]
    masks = []
    for m, img in ((reference_valid, ref), (secondary_valid, sec)):
        if m is None:
            masks.append(None)
        else:
            m = np.asarray(m, dtype=bool)
            if m.shape != img.shape:
                raise ValueError(f"a mask is {m.shape} but the image is {img.shape}")
            masks.append(_mask_bytes(m))
    st, cols = points_struct(grid)
    outs = [np.empty(n, np.float32) for _ in range(3)] + [np.empty(n, np.uint16),
                                                           np.empty(n, np.uint8)]
    prm = multichip_params(p)  # holds the rotation angles the request points at
    req = _lib.ArRequest(
        arrays[0].ctypes.data, arrays[1].ctypes.data,
        masks[0].ctypes.data if masks[0] is not None else None,
        masks[1].ctypes.data if masks[1] is not None else None,
        ref.shape[0], ref.shape[1], DTYPES[ref.dtype], prepare_options(p), prm,
        ctypes.pointer(st), gr, gc, *(o.ctypes.data for o in outs))
    t = _lib._i64()
    ctx.check(ctx.lib.ar_submit(ctx.handle, ctypes.byref(req), ctypes.byref(t)))
    return Ticket(ctx, t.value, (arrays, masks, st, cols, req, prm), outs, (gr, gc))
