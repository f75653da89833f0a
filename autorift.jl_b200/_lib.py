"""ctypes binding of libautorift_gpu.so (include/autorift_gpu.h).

The library is the only compute path: if it is missing or no GPU is visible, every call that
would compute raises. There is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import threading
import weakref
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libautorift_gpu.so"

AR_OK, AR_ERR_ARG, AR_ERR_SIZE, AR_ERR_OOM, AR_ERR_TIMEOUT, AR_ERR_CUDA, AR_ERR_UNSUPPORTED = range(7)
AR_U8, AR_U16, AR_F32, AR_I16, AR_F64 = range(5)
AR_ZNCC, AR_NCC = 0, 1

# Every symbol include/autorift_gpu.h declares, with (restype, argtypes).
_p = ctypes.c_void_p
_i32 = ctypes.c_int
_i64 = ctypes.c_int64
_sz = ctypes.c_size_t


class ArPrepareOpts(ctypes.Structure):
    """`ar_prepare_opts`: preprocess method and width, Wallis floor, quantisation."""

    _fields_ = [("preprocess", _i32), ("width", _i32), ("min_std", ctypes.c_double),
                ("quantize", _i32)]


class ArMultichipParams(ctypes.Structure):
    """`ar_multichip_params`: the Params fields correlate_multichip reads."""

    _fields_ = [("chip_size_base", _i32), ("chip_size_min", _i32), ("chip_size_max", _i32),
                ("chip_aspect", ctypes.c_double), ("min_search_radius", _i32),
                ("coarse_stride", _i32), ("coarse_buffer", _i32),
                ("min_coarse_valid_fraction", ctypes.c_double), ("upsampling", _i32),
                ("measure", _i32), ("outliers", _i32), ("outlier_window", _i32),
                ("outlier_iterations", _i32), ("min_agree_fraction", ctypes.c_double),
                ("agree_tolerance", ctypes.c_double), ("mad_scale", ctypes.c_double),
                ("fill_window", _i32), ("rotation_count", _i32), ("rotation_angles", _p),
                ("level_measure_count", _i32), ("level_measures", _i32 * 8)]


class ArPoints(ctypes.Structure):
    """`ar_points`: the eight PointSet fields (src/points.jl:50-74) plus the count."""

    _fields_ = [("x", _p), ("y", _p), ("radius_x", _p), ("radius_y", _p),
                ("dx_prior", _p), ("dy_prior", _p), ("chip_size_x", _p), ("chip_size_y", _p),
                ("n", _i64)]


class ArRequest(ctypes.Structure):
    """`ar_request` (include/autorift_gpu.h): one autorift() request for the request loop."""

    _fields_ = [("reference", _p), ("secondary", _p), ("reference_valid", _p),
                ("secondary_valid", _p), ("nrows", _i64), ("ncols", _i64),
                ("dtype", ctypes.c_int), ("prepare", ArPrepareOpts),
                ("params", ArMultichipParams), ("grid", ctypes.POINTER(ArPoints)),
                ("grid_rows", _i64), ("grid_cols", _i64), ("dx", _p), ("dy", _p),
                ("correlation", _p), ("chip_size", _p), ("interpolated", _p)]


AR_PRE_NONE, AR_PRE_HIGHPASS, AR_PRE_WALLIS = 0, 1, 2
AR_OPT_TENSOR_CORES, AR_OPT_SERVE_SLOTS, AR_OPT_SERVE_MEMORY_MB, AR_OPT_SPLIT_BF16 = 1, 2, 3, 4
AR_OPT_AUTOTUNE, AR_OPT_SHAPE_BINS, AR_OPT_UINT8_KERNEL = 5, 6, 7
AR_QUANT_NONE, AR_QUANT_UINT8 = 0, 1


SIGNATURES = {
    "ar_version": (_i32, []),
    "ar_ctx_create": (_i32, [_i32, ctypes.POINTER(_p)]),
    "ar_ctx_destroy": (_i32, [_p]),
    "ar_last_error": (_i32, [_p, ctypes.c_char_p, _sz]),
    "ar_pair_upload": (_i32, [_p, _p, _p, _p, _p, _i64, _i64, _i32, ctypes.POINTER(_p)]),
    "ar_pair_destroy": (_i32, [_p]),
    "ar_prepare": (_i32, [_p, _p, ctypes.POINTER(ArPrepareOpts), ctypes.POINTER(_p)]),
    "ar_pair_download": (_i32, [_p, _p, _p, _p, _p, _p]),
    "ar_pair_info": (_i32, [_p, ctypes.POINTER(_i32), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "ar_track": (_i32, [_p, _p, ctypes.POINTER(ArPoints), _i32, _i32, _p, _p, _p, _p]),
    "ar_track_rotated": (_i32, [_p, _p, ctypes.POINTER(ArPoints), _i32, _i32, _p, _i32, _p, _p,
                                _p, _p]),
    "ar_track_device": (_i32, [_p, _p, ctypes.POINTER(ArPoints), _i32, _i32, _p, _p, _p, _p, _p]),
    "ar_track_device_rotated": (_i32, [_p, _p, ctypes.POINTER(ArPoints), _i32, _i32, _p, _i32,
                                       _p, _p, _p, _p, _p]),
    "ar_track_device_static": (_i32, [_p, _p, _p, _i64, _i64, _i32, ctypes.POINTER(ArPoints), _i32,
                                      _i32, _p, _p, _p, _p, _p, ctypes.c_char_p, _sz]),
    "ar_scratch_allocations": (_i32, [ctypes.POINTER(_i64)]),
    "ar_correlate": (_i32, [_p, _p, _p, _i32, _i64, _i64, _i64, _i64, _i32, _p,
                            ctypes.POINTER(_i32)]),
    "ar_refine_patches": (_i32, [_p, _p, _i64, _i32, _p, _p, _p]),
    "ar_multichip": (_i32, [_p, _p, ctypes.POINTER(ArPoints), _i64, _i64,
                            ctypes.POINTER(ArMultichipParams), _p, _p, _p, _p, _p]),
    "ar_multichip_device": (_i32, [_p, _p, ctypes.POINTER(ArPoints), _i64, _i64,
                                   ctypes.POINTER(ArMultichipParams), _p, _p, _p, _p, _p, _p]),
    "ar_ctx_stream": (_i32, [_p, ctypes.POINTER(_p)]),
    "ar_ctx_set_option": (_i32, [_p, ctypes.c_int, ctypes.c_int]),
    "ar_submit": (_i32, [_p, ctypes.POINTER(ArRequest), ctypes.POINTER(_i64)]),
    "ar_poll": (_i32, [_p, _i64, ctypes.POINTER(ctypes.c_int)]),
    "ar_wait": (_i32, [_p, _i64, ctypes.c_int]),
    "ar_request_times": (_i32, [_p, _i64, ctypes.POINTER(ctypes.c_double),
                                ctypes.POINTER(ctypes.c_double)]),
    "ar_release": (_i32, [_p, _i64]),
    "ar_tc_selftest": (_i32, [_p, _p, ctypes.c_int, _p, ctypes.c_int, _p, _p]),
    "ar_ctx_set_timing": (_i32, [_p, _i32]),
    "ar_kernel_times": (_i32, [_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                               ctypes.POINTER(ctypes.c_double)]),
    "ar_ctx_tuned": (_i32, [_p, _p, _i64, ctypes.POINTER(_i64)]),
    "ar_synchronize": (_i32, [_p]),
}

_lib = None
_lock = threading.Lock()


class ArError(RuntimeError):
    """A non-zero status from the library, with its message."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


def load(path: Path | None = None):
    """Load the shared library and declare every exported signature."""
    global _lib
    with _lock:
        if _lib is None:
            p = Path(path) if path else LIB_PATH
            if not p.exists():
                raise RuntimeError(
                    f"{p.name} is not built; run __graft_entry__.build() (nvcc for sm_100a). "
                    "There is no CPU fallback.")
            L = ctypes.CDLL(str(p))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


class Context:
    """An `ar_ctx` on one CUDA device (owns its stream and scratch)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = _p()
        rc = self.lib.ar_ctx_create(int(device), ctypes.byref(h))
        if rc != AR_OK:
            raise ArError(rc, f"ar_ctx_create(device={device}) failed: no usable CUDA device")
        self.handle = h
        self.device = int(device)
        # Device pairs of this context, released before it is destroyed (a pair cannot outlive
        # its context's memory pool).
        self._pairs = weakref.WeakSet()

    def check(self, rc: int):
        if rc != AR_OK:
            buf = ctypes.create_string_buffer(512)
            self.lib.ar_last_error(self.handle, buf, 512)
            raise ArError(rc, buf.value.decode(errors="replace"))

    def set_timing(self, enable: bool):
        self.check(self.lib.ar_ctx_set_timing(self.handle, int(bool(enable))))

    def set_option(self, option: int, value: int):
        self.check(self.lib.ar_ctx_set_option(self.handle, int(option), int(value)))

    def stream(self) -> int:
        """The context's CUDA stream handle."""
        h = ctypes.c_void_p()
        self.check(self.lib.ar_ctx_stream(self.handle, ctypes.byref(h)))
        return h.value or 0

    def kernel_times(self):
        """(corr_ms, refine_ms, track_launches, kernel_launches, corr_flops) since the last
        call."""
        a, b, f = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        t, n = _i64(), _i64()
        self.check(self.lib.ar_kernel_times(self.handle, ctypes.byref(a), ctypes.byref(b),
                                            ctypes.byref(t), ctypes.byref(n), ctypes.byref(f)))
        return a.value, b.value, t.value, n.value, f.value

    def tuned(self):
        """The autotuner's choices so far: one dict per pass geometry (largest chip rows and
        columns, surface rows and columns) with the kernel kept ("k_corr_tc2", "k_corr_tc" or
        "k_corr")."""
        cnt = _i64()
        self.check(self.lib.ar_ctx_tuned(self.handle, None, 0, ctypes.byref(cnt)))
        buf = (ctypes.c_int32 * (5 * max(cnt.value, 1)))()
        self.check(self.lib.ar_ctx_tuned(self.handle, buf, cnt.value, ctypes.byref(cnt)))
        names = {2: "k_corr_tc2", 1: "k_corr_tc", 0: "k_corr"}
        return [{"chip": [buf[5 * i], buf[5 * i + 1]], "surface": [buf[5 * i + 2], buf[5 * i + 3]],
                 "kernel": names.get(buf[5 * i + 4], str(buf[5 * i + 4]))}
                for i in range(cnt.value)]

    def close(self):
        if getattr(self, "handle", None):
            for pair in list(getattr(self, "_pairs", ())):
                pair.release()
            self.lib.ar_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = {}


def default_context(device: int = 0) -> Context:
    """One shared context per device for the convenience API."""
    with _lock:
        ctx = _default_ctx.get(device)
    if ctx is None:
        ctx = Context(device)
        with _lock:
            _default_ctx.setdefault(device, ctx)
            ctx = _default_ctx[device]
    return ctx
