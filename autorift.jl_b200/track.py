"""The grid pass on the GPU: ImagePair, DisplacementField and track (src/track.jl).

`track(pair, pts, p)` is the drop-in for `track!`/`track`: the same point semantics (the +0.5
grid offset, the asymmetric window, zero padding only when some window leaves the image, the
valid-chip gate), the same outputs (dx, dy, correlation NaN where there is no measurement,
searched), computed by libautorift_gpu through its C ABI.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .methods import (NCC, NoRefine, Params, RotationSearch, ZNCC, angles, params as make_params,
                      upsampling)
from .points import FIELDS, PointSet

DTYPES = {np.dtype(np.uint8): _lib.AR_U8, np.dtype(np.uint16): _lib.AR_U16,
          np.dtype(np.float32): _lib.AR_F32, np.dtype(np.int16): _lib.AR_I16}


def _colmajor(a, dtype=None) -> np.ndarray:
    a = np.asarray(a) if dtype is None else np.asarray(a, dtype=dtype)
    return np.asfortranarray(a)


def _mask_bytes(m) -> np.ndarray:
    """A validity mask as the column-major bytes the C ABI reads: a bool array is viewed as
    its bytes (0/1) without a copy when it is already column-major."""
    m = np.asarray(m)
    if m.dtype == np.bool_:
        return np.asfortranarray(m).view(np.uint8)
    return _colmajor(m != 0).view(np.uint8)


class ImagePair:
    """The two images to correlate with their validity masks (src/preprocess.jl:41-106).

    Masks default to finiteness; zero is a valid value unless a mask says otherwise. The pair
    is uploaded to the device on first use and kept there.
    """

    def __init__(self, reference, secondary, reference_valid=None, secondary_valid=None):
        ref = np.asarray(reference)
        sec = np.asarray(secondary)
        if ref.shape != sec.shape:
            raise ValueError(f"reference is {ref.shape} but secondary is {sec.shape}; the two "
                             "images must be co-registered to a common grid before correlation")
        if ref.ndim != 2:
            raise ValueError("images must be matrices")
        if sec.dtype != ref.dtype:
            sec = sec.astype(ref.dtype)
        self.reference = ref
        self.secondary = sec
        # Masks the caller gave (None: the default, finiteness, which the device computes).
        self.given_reference_valid = self._mask(reference_valid, ref, "reference_valid")
        self.given_secondary_valid = self._mask(secondary_valid, sec, "secondary_valid")
        self._device = {}

    @staticmethod
    def _mask(m, img, name):
        if m is None:
            return None
        m = np.asarray(m, dtype=bool)
        if m.shape != img.shape:
            raise ValueError(f"{name} is {m.shape} but the image is {img.shape}")
        return m

    @staticmethod
    def _default(img):
        return np.isfinite(img) if img.dtype.kind in "fc" else np.ones(img.shape, bool)

    @property
    def reference_valid(self) -> np.ndarray:
        m = self.given_reference_valid
        return self._default(self.reference) if m is None else m

    @property
    def secondary_valid(self) -> np.ndarray:
        m = self.given_secondary_valid
        return self._default(self.secondary) if m is None else m

    @property
    def shape(self):
        return self.reference.shape

    @property
    def dtype(self):
        return self.reference.dtype

    def valid(self) -> np.ndarray:
        return self.reference_valid & self.secondary_valid

    def device(self, ctx: "_lib.Context"):
        """The `ar_pair` handle on ctx's device (uploaded once)."""
        h = self._device.get(id(ctx))
        if h is not None:
            return h
        if self.dtype not in DTYPES:
            raise TypeError(f"element type {self.dtype} is not supported by the GPU correlator "
                            f"(supported: {', '.join(str(d) for d in DTYPES)})")
        ref = _colmajor(self.reference)
        sec = _colmajor(self.secondary)
        # A mask left to its default is not uploaded: the device evaluates the same finiteness
        # test (ar_pair_upload with a NULL mask).
        rv, sv = (None if m is None else _mask_bytes(m)
                  for m in (self.given_reference_valid, self.given_secondary_valid))
        out = ctypes.c_void_p()
        ctx.check(ctx.lib.ar_pair_upload(ctx.handle, ref.ctypes.data, sec.ctypes.data,
                                         None if rv is None else rv.ctypes.data,
                                         None if sv is None else sv.ctypes.data, ref.shape[0],
                                         ref.shape[1], DTYPES[self.dtype], ctypes.byref(out)))
        h = _DevicePair(ctx, out)
        self._device[id(ctx)] = h
        return h


class _DevicePair:
    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.handle = handle
        ctx._pairs.add(self)

    def release(self):
        """Destroy the device pair (idempotent; a closed context already freed it)."""
        if self.handle and getattr(self.ctx, "handle", None):
            self.ctx.lib.ar_pair_destroy(self.handle)
        self.handle = None

    def info(self):
        dt = ctypes.c_int()
        nr = ctypes.c_int64()
        nc = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.ar_pair_info(self.handle, ctypes.byref(dt), ctypes.byref(nr),
                                                 ctypes.byref(nc)))
        return dt.value, (nr.value, nc.value)

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


_NP_OF = {_lib.AR_U8: np.uint8, _lib.AR_U16: np.uint16, _lib.AR_F32: np.float32,
          _lib.AR_I16: np.int16}


class PreparedPair:
    """A filtered and quantised pair resident on the device: the `prepared` ImagePair of the
    reference's Cache (src/api.jl:30-44), produced by `prepare`."""

    def __init__(self, dev: _DevicePair):
        self._dev = dev
        self.dtype_code, self.shape = dev.info()
        self.dtype = np.dtype(_NP_OF[self.dtype_code])

    def device(self, ctx):
        if ctx is not self._dev.ctx:
            raise ValueError("the prepared pair belongs to another context")
        return self._dev

    def download(self):
        """(reference, secondary, reference_valid, secondary_valid) as host arrays."""
        nr, nc = self.shape
        out = [np.empty((nr, nc), self.dtype, order="F") for _ in range(2)]
        masks = [np.empty((nr, nc), np.uint8, order="F") for _ in range(2)]
        ctx = self._dev.ctx
        ctx.check(ctx.lib.ar_pair_download(ctx.handle, self._dev.handle, out[0].ctypes.data,
                                           out[1].ctypes.data, masks[0].ctypes.data,
                                           masks[1].ctypes.data))
        return out[0], out[1], masks[0].astype(bool), masks[1].astype(bool)


def prepare_options(p: Params) -> "_lib.ArPrepareOpts":
    """The `ar_prepare_opts` of a parameter set's preprocess and quantize methods."""
    from .methods import Highpass, NoPreprocess, NoQuantize, QuantizeUInt8, Wallis
    pre = p.preprocess
    if isinstance(pre, NoPreprocess):
        kind, width, floor = _lib.AR_PRE_NONE, 0, 0.0
    elif isinstance(pre, Highpass):
        kind, width, floor = _lib.AR_PRE_HIGHPASS, pre.width, 0.0
    elif isinstance(pre, Wallis):
        kind, width, floor = _lib.AR_PRE_WALLIS, pre.width, pre.min_std
    else:
        raise ValueError(f"{type(pre).__name__} has no GPU implementation")
    q = _lib.AR_QUANT_UINT8 if isinstance(p.quantize, QuantizeUInt8) else _lib.AR_QUANT_NONE
    return _lib.ArPrepareOpts(kind, width, float(floor), q)


def prepare(pair: ImagePair, p: Params | None = None, ctx=None) -> PreparedPair:
    """Filter and quantise a pair on the device (`_prepare`, src/api.jl:305-311)."""
    p = p if p is not None else make_params()
    ctx = ctx or _lib.default_context()
    raw = pair.device(ctx)
    out = ctypes.c_void_p()
    opts = prepare_options(p)
    ctx.check(ctx.lib.ar_prepare(ctx.handle, raw.handle, ctypes.byref(opts), ctypes.byref(out)))
    return PreparedPair(_DevicePair(ctx, out))


@dataclass
class DisplacementField:
    """Per-point results of a pass (src/track.jl:46-62)."""

    dx: np.ndarray
    dy: np.ndarray
    correlation: np.ndarray
    searched: np.ndarray

    @property
    def shape(self):
        return self.dx.shape

    def __len__(self):
        return int(self.dx.size)


def displacement_field(pts: PointSet) -> DisplacementField:
    sz = pts.shape
    return DisplacementField(np.full(sz, np.nan, np.float32), np.full(sz, np.nan, np.float32),
                             np.full(sz, np.nan, np.float32), np.zeros(sz, bool))


def nmeasured(d) -> int:
    return int(np.count_nonzero(~np.isnan(d.dx)))


def points_struct(pts: PointSet):
    """`ar_points` over host arrays; returns (struct, keepalive)."""
    cols = {n: pts.flat(n) for n in FIELDS}
    s = _lib.ArPoints(*(c.ctypes.data for c in (cols[n] for n in FIELDS)), len(pts))
    return s, cols


def _measure_code(m) -> int:
    if isinstance(m, ZNCC):
        return _lib.AR_ZNCC
    if isinstance(m, NCC):
        return _lib.AR_NCC
    raise ValueError("`Coherence` needs complex input; the GPU correlator handles real imagery "
                     "with :zncc or :ncc")


def rotation_angles(p: Params):
    """The chip rotations of `p.rotation` as a float64 array, or None for NoRotationSearch."""
    if isinstance(p.rotation, RotationSearch):
        return np.ascontiguousarray(angles(p.rotation), dtype=np.float64)
    return None


def track(pair, pts: PointSet, p: Params | None = None, *, subpixel=None,
          measure=None, ctx: "_lib.Context | None" = None) -> DisplacementField:
    """Correlate `pair` (an ImagePair, uploaded on first use, or a PreparedPair already on the
    device) at every searchable point of `pts` (src/track.jl:103-160), with `p.rotation`'s
    chip-rotation search when it is a RotationSearch (src/track.jl:313-409)."""
    p = p if p is not None else make_params()
    sub = p.subpixel if subpixel is None else subpixel
    meas = p.similarity[0] if measure is None else measure
    ctx = ctx or _lib.default_context()
    n = len(pts)
    out = displacement_field(pts)
    if n == 0:
        return out
    dp = pair.device(ctx)
    s, keep = points_struct(pts)
    dx = np.empty(n, np.float32)
    dy = np.empty(n, np.float32)
    corr = np.empty(n, np.float32)
    searched = np.empty(n, np.uint8)
    rot = rotation_angles(p)
    if rot is None:
        ctx.check(ctx.lib.ar_track(ctx.handle, dp.handle, ctypes.byref(s), upsampling(sub),
                                   _measure_code(meas), dx.ctypes.data, dy.ctypes.data,
                                   corr.ctypes.data, searched.ctypes.data))
    else:
        ctx.check(ctx.lib.ar_track_rotated(ctx.handle, dp.handle, ctypes.byref(s),
                                           upsampling(sub), _measure_code(meas),
                                           rot.ctypes.data, rot.size, dx.ctypes.data,
                                           dy.ctypes.data, corr.ctypes.data,
                                           searched.ctypes.data))
    shp = pts.shape
    out.dx = dx.reshape(shp, order="F")
    out.dy = dy.reshape(shp, order="F")
    out.correlation = corr.reshape(shp, order="F")
    out.searched = searched.astype(bool).reshape(shp, order="F")
    return out


def correlate(search, chip, radius, measure=ZNCC(), ctx=None):
    """One surface (correlate!, src/correlate.jl:528-557): returns (surface, degenerate)."""
    ctx = ctx or _lib.default_context()
    rx, ry = (radius, radius) if np.isscalar(radius) else radius
    chip = _colmajor(chip)
    search = _colmajor(search, chip.dtype)
    if chip.dtype not in DTYPES:
        raise TypeError(f"unsupported element type {chip.dtype}")
    ch, cw = chip.shape
    if search.shape != (ch + 2 * ry - 1, cw + 2 * rx - 1):
        raise ValueError(f"search window is {search.shape} but a {ch}x{cw} chip with radius "
                         f"({rx}, {ry}) requires {(ch + 2 * ry - 1, cw + 2 * rx - 1)}")
    surf = np.empty((2 * ry, 2 * rx), np.float32, order="F")
    deg = ctypes.c_int(0)
    ctx.check(ctx.lib.ar_correlate(ctx.handle, search.ctypes.data, chip.ctypes.data,
                                   DTYPES[chip.dtype], ch, cw, rx, ry, _measure_code(measure),
                                   surf.ctypes.data, ctypes.byref(deg)))
    return surf, bool(deg.value)


def refine_patches(patches, up: int, ctx=None):
    """Run the pyrUp cascade on 5x5 patches; returns (row, col, value) of each upsampled peak."""
    ctx = ctx or _lib.default_context()
    P = np.asarray(patches, dtype=np.float32)
    if P.ndim == 2:
        P = P[None]
    count = P.shape[0]
    flat = np.ascontiguousarray(np.stack([np.asfortranarray(q).ravel(order="F") for q in P]))
    row = np.empty(count, np.int32)
    col = np.empty(count, np.int32)
    val = np.empty(count, np.float32)
    ctx.check(ctx.lib.ar_refine_patches(ctx.handle, flat.ctypes.data, count, int(up),
                                        row.ctypes.data, col.ctypes.data, val.ctypes.data))
    return row, col, val
