"""ctypes binding for the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (``oracle/oracle.cpp``) restates AutoRIFT.jl's correlator on the CPU. Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may load it; the product
path never does.

All arrays are numpy arrays in *Julia* orientation: a matrix of shape ``(nrows, ncols)`` stored
column-major (``np.asfortranarray``). Point-set fields are flat vectors.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle_ar.so"

DTYPE_CODES = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.float32): 2,
               np.dtype(np.int16): 3, np.dtype(np.float64): 4}
MEASURES = {"zncc": 0, "ncc": 1}

_lib = None


def build(force: bool = False) -> Path:
    """Compile the oracle with its Makefile (g++, OpenMP, no FP contraction)."""
    if force or not _LIB_PATH.exists() or (
            _LIB_PATH.stat().st_mtime < (_HERE / "oracle.cpp").stat().st_mtime):
        subprocess.run(["make", "-B" if force else "all"], cwd=_HERE, check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(_LIB_PATH))
        p, i64, i32, f64p = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p
        L.or_correlate.argtypes = [p, p, i32, i64, i64, i64, i64, i32, p]
        L.or_correlate.restype = i32
        L.or_peak_index.argtypes = [p, i64, i64, p, p]
        L.or_peak_index.restype = None
        L.or_pyrup.argtypes = [p, i64, i64, p]
        L.or_pyrup.restype = None
        L.or_subpixel_peak.argtypes = [p, i64, i64, i64, i64, i32, f64p, f64p, p]
        L.or_subpixel_peak.restype = None
        L.or_track.argtypes = ([p, p, p, p, i64, i64, i32] + [p] * 8 + [i64, i32, i32] + [p] * 4
                               + [i32, p, i32])
        L.or_track.restype = i32
        L.or_prepare.argtypes = [p, p, i64, i64, i32, i32, i64, ctypes.c_double, i32, p, p]
        L.or_prepare.restype = i32
        L.or_multichip.argtypes = ([p, p, p, p, i64, i64, i32] + [p] * 6 + [i64, i64, p] + [p] * 5
                                   + [i32, p, i32])
        L.or_rotate_chip.argtypes = [p, i32, i64, i64, ctypes.c_double, p]
        L.or_rotate_chip.restype = i32
        L.or_multichip.restype = i32
        L.or_reject_outliers.argtypes = [p, p, p, p, p, i64, i64, i32, i32, i64, i64,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, p]
        L.or_reject_outliers.restype = i32
        L.or_max_threads.argtypes = []
        L.or_max_threads.restype = i32
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f(a, dtype=None):
    a = np.asarray(a) if dtype is None else np.asarray(a, dtype=dtype)
    return np.asfortranarray(a)


def correlate(search, chip, radius, measure: str = "zncc"):
    """Surface of ``chip`` against ``search`` (src/correlate.jl:528-557).

    Returns ``(surface, degenerate)``; ``surface`` is ``(2ry, 2rx)`` float32.
    """
    rx, ry = (radius, radius) if np.isscalar(radius) else radius
    chip = _f(chip)
    search = _f(search, chip.dtype)
    ch, cw = chip.shape
    if search.shape != (ch + 2 * ry - 1, cw + 2 * rx - 1):
        raise ValueError(f"search window is {search.shape}, expected "
                         f"{(ch + 2 * ry - 1, cw + 2 * rx - 1)}")
    out = np.empty((2 * ry, 2 * rx), dtype=np.float32, order="F")
    rc = lib().or_correlate(_ptr(search), _ptr(chip), DTYPE_CODES[chip.dtype], ch, cw, rx, ry,
                            MEASURES[measure], _ptr(out))
    if rc < 0:
        raise ValueError("unsupported dtype")
    return out, rc == 1


def peak_index(surface):
    """Row-major first strict maximum, 0-based (src/peak.jl:32-61)."""
    s = _f(surface, np.float32)
    i = ctypes.c_int64()
    j = ctypes.c_int64()
    lib().or_peak_index(_ptr(s), s.shape[0], s.shape[1], ctypes.byref(i), ctypes.byref(j))
    return i.value, j.value


def pyrup(src):
    """One pyrUp step (src/peak.jl:196-294)."""
    s = _f(src, np.float32)
    out = np.empty((2 * s.shape[0], 2 * s.shape[1]), dtype=np.float32, order="F")
    lib().or_pyrup(_ptr(s), s.shape[0], s.shape[1], _ptr(out))
    return out


def subpixel_peak(surface, radius, upsampling):
    """(dx, dy, correlation) at 1/upsampling pixel (src/peak.jl:456-522)."""
    rx, ry = (radius, radius) if np.isscalar(radius) else radius
    s = _f(surface, np.float32)
    dx = ctypes.c_double()
    dy = ctypes.c_double()
    v = np.zeros(1, dtype=np.float32)
    lib().or_subpixel_peak(_ptr(s), s.shape[0], s.shape[1], rx, ry, int(upsampling),
                           ctypes.byref(dx), ctypes.byref(dy), _ptr(v))
    return dx.value, dy.value, float(v[0])


def _angles(angles):
    """(pointer, count) of a rotation-search angle list; None or empty is NoRotationSearch."""
    if angles is None or len(angles) == 0:
        return None, 0, None
    a = np.ascontiguousarray(np.asarray(angles, dtype=np.float64).ravel())
    return _ptr(a), int(a.size), a


def rotate_chip(chip, deg: float):
    """_rotate_chip (src/track.jl:377-409): the chip turned by ``deg`` degrees, Float32."""
    c = _f(chip)
    ch, cw = c.shape
    out = np.empty((ch, cw), dtype=np.float32, order="F")
    rc = lib().or_rotate_chip(_ptr(c), DTYPE_CODES[c.dtype], ch, cw, float(deg), _ptr(out))
    if rc != 0:
        raise ValueError("unsupported dtype")
    return out


def track(reference, secondary, points, upsampling: int = 64, measure: str = "zncc",
          reference_valid=None, secondary_valid=None, nthreads: int = 0, angles=None):
    """track! over a point set (src/track.jl:103-152).

    ``points`` is a mapping with the eight PointSet fields ``x, y, radius_x, radius_y,
    dx_prior, dy_prior, chip_size_x, chip_size_y`` (any shape; flattened column-major).
    ``angles`` (degrees, the reference's ``angles(RotationSearch)``) turns on the rotation
    search (src/track.jl:313-350). Returns ``(dx, dy, correlation, searched)`` as flat arrays.
    """
    ref = _f(reference)
    sec = _f(secondary, ref.dtype)
    if ref.shape != sec.shape:
        raise ValueError("reference and secondary differ in shape")
    nrows, ncols = ref.shape
    if reference_valid is None:
        reference_valid = np.isfinite(ref) if ref.dtype.kind == "f" else np.ones(ref.shape, bool)
    if secondary_valid is None:
        secondary_valid = np.isfinite(sec) if sec.dtype.kind == "f" else np.ones(sec.shape, bool)
    rv = _f(reference_valid, np.uint8)
    sv = _f(secondary_valid, np.uint8)

    def fld(name, dt):
        return np.ascontiguousarray(np.asarray(points[name], dtype=dt).ravel(order="F"))

    x, y = fld("x", np.float64), fld("y", np.float64)
    rx, ry = fld("radius_x", np.int64), fld("radius_y", np.int64)
    dx0, dy0 = fld("dx_prior", np.float64), fld("dy_prior", np.float64)
    csx, csy = fld("chip_size_x", np.int64), fld("chip_size_y", np.int64)
    n = x.size
    dx = np.empty(n, np.float32)
    dy = np.empty(n, np.float32)
    corr = np.empty(n, np.float32)
    searched = np.empty(n, np.uint8)
    rc = lib().or_track(_ptr(ref), _ptr(sec), _ptr(rv), _ptr(sv), nrows, ncols,
                        DTYPE_CODES[ref.dtype], _ptr(x), _ptr(y), _ptr(rx), _ptr(ry),
                        _ptr(dx0), _ptr(dy0), _ptr(csx), _ptr(csy), n, int(upsampling),
                        MEASURES[measure], _ptr(dx), _ptr(dy), _ptr(corr), _ptr(searched),
                        int(nthreads), *_angles(angles)[:2])
    if rc != 0:
        raise ValueError(f"or_track failed with {rc}")
    return dx, dy, corr, searched.astype(bool)


PREPROCESS = {"none": 0, "highpass": 1, "wallis": 2}
QUANTIZE = {"none": 0, "uint8": 1}


def prepare(img, mask=None, preprocess: str = "highpass", width: int = 5, min_std: float = 0.0,
            quantize: str = "uint8"):
    """preprocess then quantize one image (src/api.jl:305-306): returns (image, mask)."""
    a = _f(img)
    nr, nc = a.shape
    m = None if mask is None else _f(mask, np.uint8)
    pre, q = PREPROCESS[preprocess], QUANTIZE[quantize]
    odt = np.uint8 if q == 1 else (np.float32 if pre else a.dtype)
    out = np.empty((nr, nc), dtype=odt, order="F")
    vout = np.empty((nr, nc), dtype=np.uint8, order="F")
    rc = lib().or_prepare(_ptr(a), _ptr(m) if m is not None else None, nr, nc,
                          DTYPE_CODES[a.dtype], pre, int(width), float(min_std), q, _ptr(out),
                          _ptr(vout))
    if rc != 0:
        raise ValueError("unsupported dtype")
    return out, vout.astype(bool)


def multichip(reference, secondary, grid, params: dict, reference_valid=None,
              secondary_valid=None, nthreads: int = 0, angles=None):
    """correlate_multichip (src/multichip.jl:106-137) over a gridded point set.

    ``grid`` maps the PointSet fields to (gr, gc) arrays; ``params`` holds chip_base, chip_min,
    chip_max, aspect, min_radius, stride, buffer, min_frac, up, measure (0/1), outliers (0/1),
    window, iterations, min_agree_fraction, agree_tolerance, mad_scale, fill_window, and
    optionally ``level_measures`` (0/1 per chip-size level, the last repeating).
    ``angles`` turns on the rotation search at every level, as in ``track``.
    Returns (dx, dy, correlation, chip_size, interpolated) as (gr, gc) arrays.
    """
    ref = _f(reference)
    sec = _f(secondary, ref.dtype)
    nrows, ncols = ref.shape
    if reference_valid is None:
        reference_valid = np.isfinite(ref) if ref.dtype.kind == "f" else np.ones(ref.shape, bool)
    if secondary_valid is None:
        secondary_valid = np.isfinite(sec) if sec.dtype.kind == "f" else np.ones(sec.shape, bool)
    rv = _f(reference_valid, np.uint8)
    sv = _f(secondary_valid, np.uint8)
    gr, gc = np.shape(grid["x"])

    def fld(name, dt):
        return np.ascontiguousarray(np.asarray(grid[name], dtype=dt).ravel(order="F"))

    keys = ["chip_base", "chip_min", "chip_max", "aspect", "min_radius", "stride", "buffer",
            "min_frac", "up", "measure", "outliers", "window", "iterations",
            "min_agree_fraction", "agree_tolerance", "mad_scale", "fill_window"]
    lev = list(params.get("level_measures", ()))
    if len(lev) > 8:
        raise ValueError("at most 8 per-level measures")
    prm = np.array([float(params[k]) for k in keys] + [float(len(lev))]
                   + [float(v) for v in lev] + [0.0] * (8 - len(lev)), dtype=np.float64)
    cols = [fld("x", np.float64), fld("y", np.float64), fld("radius_x", np.int64),
            fld("radius_y", np.int64), fld("dx_prior", np.float64), fld("dy_prior", np.float64)]
    n = gr * gc
    dx = np.empty(n, np.float32)
    dy = np.empty(n, np.float32)
    c = np.empty(n, np.float32)
    cs = np.empty(n, np.uint16)
    it = np.empty(n, np.uint8)
    rc = lib().or_multichip(_ptr(ref), _ptr(sec), _ptr(rv), _ptr(sv), nrows, ncols,
                            DTYPE_CODES[ref.dtype], *[_ptr(a) for a in cols], gr, gc, _ptr(prm),
                            _ptr(dx), _ptr(dy), _ptr(c), _ptr(cs), _ptr(it), int(nthreads),
                            *_angles(angles)[:2])
    if rc != 0:
        raise ValueError("unsupported dtype")
    shp = lambda a: a.reshape((gr, gc), order="F")
    return shp(dx), shp(dy), shp(c), shp(cs), shp(it).astype(bool)


def reject_outliers(dx, dy, rx, ry, valid, up: int, outliers: str = "gardner", window: int = 5,
                    iterations: int = 3, min_agree_fraction: float = 8 / 25,
                    agree_tolerance: float = 0.2, mad_scale: float = 4.0):
    """reject_outliers (src/outliers.jl:38-160) on (nr, nc) fields: the keep mask."""
    dx = _f(dx, np.float32)
    nr, nc = dx.shape
    keep = np.empty((nr, nc), np.uint8, order="F")
    lib().or_reject_outliers(_ptr(dx), _ptr(_f(dy, np.float32)), _ptr(_f(rx, np.int64)),
                             _ptr(_f(ry, np.int64)), _ptr(_f(valid, np.uint8)), nr, nc, int(up),
                             1 if outliers == "gardner" else 0, window, iterations,
                             min_agree_fraction, agree_tolerance, mad_scale, _ptr(keep))
    return keep.astype(bool)


def max_threads() -> int:
    return int(lib().or_max_threads())


if os.environ.get("AUTORIFT_ORACLE_REBUILD"):
    build(force=True)
