"""Method objects and the resolved parameter set (src/types.jl, src/params.jl).

The reference maps every keyword Symbol to a singleton or small struct in one file
(src/params.jl:12-47) and validates numbers once, at the API boundary. This module mirrors
that contract: `params(**kw)` returns a frozen `Params` whose fields are method objects, with
the reference's defaults and its error cases (raised as ValueError, the Python spelling of
Julia's ArgumentError).
"""

from __future__ import annotations

import math
import numbers
from dataclasses import dataclass, field
from typing import Tuple


# ---------------------------------------------------------------------------------------------
# Similarity measures (src/types.jl:66-205)

@dataclass(frozen=True)
class ZNCC:
    code = 0


@dataclass(frozen=True)
class NCC:
    code = 1


@dataclass(frozen=True)
class Coherence:
    code = 2


# ---------------------------------------------------------------------------------------------
# Sub-pixel refinement (src/types.jl:207-257)

@dataclass(frozen=True)
class NoRefine:
    upsampling: int = 1


@dataclass(frozen=True)
class PyramidRefine:
    upsampling: int = 64

    def __post_init__(self):
        up = self.upsampling
        if not isinstance(up, (int,)) or isinstance(up, bool):
            raise ValueError(f"`upsampling` must be an integer, got {up!r}")
        if up <= 1:
            raise ValueError(f"`upsampling` must be > 1, got {up}")
        if up & (up - 1):
            raise ValueError(f"`upsampling` must be a power of 2, got {up}")


def upsampling(m) -> int:
    """The sub-pixel quantisation denominator (src/types.jl:255-257)."""
    return 1 if isinstance(m, NoRefine) else m.upsampling


# ---------------------------------------------------------------------------------------------
# Preprocessing (src/types.jl:259-378)

def _check_filter_width(width: int, who: str) -> int:
    if width < 3:
        raise ValueError(f"{who} `width` must be >= 3, got {width}")
    if width % 2 == 0:
        raise ValueError(f"{who} `width` must be odd so the filter has a well-defined centre, "
                         f"got {width}")
    return int(width)


@dataclass(frozen=True)
class NoPreprocess:
    pass


@dataclass(frozen=True)
class Highpass:
    width: int = 5

    def __post_init__(self):
        _check_filter_width(self.width, "Highpass")


@dataclass(frozen=True)
class Wallis:
    width: int = 5
    min_std: float = 0.0

    def __post_init__(self):
        if self.min_std < 0:
            raise ValueError(f"`min_std` must be >= 0, got {self.min_std}")
        _check_filter_width(self.width, "Wallis")


def filter_width(m) -> int:
    return getattr(m, "width", 0)


# ---------------------------------------------------------------------------------------------
# Quantisation (src/types.jl:466-499)

@dataclass(frozen=True)
class QuantizeUInt8:
    pass


@dataclass(frozen=True)
class NoQuantize:
    pass


# ---------------------------------------------------------------------------------------------
# Outlier rejection (src/types.jl:505-700)

@dataclass(frozen=True)
class GardnerFilter:
    window: int = 5
    iterations: int = 3
    min_agree_fraction: float = 8 / 25
    agree_tolerance: float = 0.2
    mad_scale: float = 4.0

    def __post_init__(self):
        if self.window % 2 == 0:
            raise ValueError("outlier filter `window` must be odd so the neighbourhood has a "
                             f"centre, got {self.window}")
        if self.window < 3:
            raise ValueError(f"outlier filter `window` must be >= 3, got {self.window}")
        if self.iterations < 1:
            raise ValueError(f"outlier filter `iterations` must be >= 1, got {self.iterations}")
        if not (0 <= self.min_agree_fraction <= 1):
            raise ValueError("`min_agree_fraction` must be in [0, 1], got "
                             f"{self.min_agree_fraction}")
        if not (0 < self.agree_tolerance <= 1):
            raise ValueError("`agree_tolerance` must be in [0, 1] and non-zero, got "
                             f"{self.agree_tolerance}")
        if not self.mad_scale > 0:
            raise ValueError(f"`mad_scale` must be positive, got {self.mad_scale}")


@dataclass(frozen=True)
class NoOutlierFilter:
    pass


def window(m) -> int:
    """Neighbourhood width an outlier method needs (src/types.jl:680-681)."""
    return m.window if isinstance(m, GardnerFilter) else 0


def relax(m):
    """The coarse-pass variant of a method (src/types.jl:699-703)."""
    if isinstance(m, GardnerFilter):
        return GardnerFilter(window=m.window, iterations=max(m.iterations - 1, 1),
                             min_agree_fraction=m.min_agree_fraction,
                             agree_tolerance=m.agree_tolerance, mad_scale=m.mad_scale)
    return m


@dataclass(frozen=True)
class NoRotationSearch:
    """Rotation search off (src/types.jl:507-527): one correlation per point."""


MAX_ROTATION_ANGLES = 64  # AR_MAX_ROTATION_ANGLES of the C-ABI


@dataclass(frozen=True, init=False)
class RotationSearch:
    """Per-chip rotation search (src/types.jl:529-557): each point correlates its chip turned by
    every angle of ``angles(m)`` (``m.angles`` minus ``m.about``, degrees) and keeps the surface
    with the strictly highest peak (src/track.jl:313-350). ``about`` centres the search on a
    scene rotation. At least one angle; angles distinct; angles and ``about`` finite; at most
    ``MAX_ROTATION_ANGLES`` (the device limit -- the reference has none)."""

    angles: Tuple[float, ...]
    about: float

    def __init__(self, angles=(-3.0, 0.0, 3.0), about=0.0):
        if isinstance(angles, (str, bytes)) or not hasattr(angles, "__iter__"):
            raise ValueError(f"`RotationSearch` angles must be a collection of real numbers, "
                             f"got a {type(angles).__name__}.")
        try:
            t = tuple(float(a) for a in angles)
        except (TypeError, ValueError):
            raise ValueError("`RotationSearch` angles must be real numbers.") from None
        if not t:
            raise ValueError("`RotationSearch` needs at least one angle; use "
                             "`NoRotationSearch()` to disable.")
        if len(set(t)) != len(t):
            raise ValueError(f"`RotationSearch` angles must be distinct, got {t} -- a repeated "
                             "angle costs a full correlation and can never win.")
        if isinstance(about, bool) or not isinstance(about, (int, float)):
            raise TypeError(f"`about` must be a real number, got a {type(about).__name__}.")
        a = float(about)
        if not (all(math.isfinite(x) for x in t) and math.isfinite(a)):
            raise ValueError(f"`RotationSearch` needs finite angles and a finite `about`, got "
                             f"angles {t} about {a}.")
        if len(t) > MAX_ROTATION_ANGLES:
            raise ValueError(f"`RotationSearch` takes at most {MAX_ROTATION_ANGLES} angles on "
                             f"the device, got {len(t)}.")
        object.__setattr__(self, "angles", t)
        object.__setattr__(self, "about", a)


def angles(m: RotationSearch) -> Tuple[float, ...]:
    """The chip rotations a pass tries, in degrees: ``m.angles .- m.about``
    (src/types.jl:577)."""
    if not isinstance(m, RotationSearch):
        raise TypeError("`angles` is defined for RotationSearch only")
    return tuple(a - m.about for a in m.angles)


def _rotation(x):
    """The rotation keyword (src/params.jl:167-180): None/False off, True the default search,
    a collection of real angles (tuple, list, range, numpy array), or a rotation method."""
    if x is None or x is False:
        return NoRotationSearch()
    if x is True:
        return RotationSearch()
    if isinstance(x, (NoRotationSearch, RotationSearch)):
        return x
    if isinstance(x, (tuple, list, range)) or (hasattr(x, "dtype") and hasattr(x, "__iter__")):
        vals = list(x)
        if all(isinstance(v, numbers.Real) for v in vals):
            return RotationSearch(vals)
    raise ValueError(f"`rotation` must be `None`, a `bool`, a collection of angles, or a "
                     f"`RotationMethod`, got a {type(x).__name__}.")


# ---------------------------------------------------------------------------------------------
# Params (src/types.jl:781-829)

@dataclass(frozen=True)
class Params:
    similarity: Tuple = (ZNCC(),)
    preprocess: object = Highpass()
    quantize: object = QuantizeUInt8()
    subpixel: object = PyramidRefine()
    outliers: object = GardnerFilter()
    threaded: bool = False
    rotation: object = NoRotationSearch()
    chip_size_base: int = 32
    chip_size_min: int = 32
    chip_size_max: int = 128
    chip_aspect: float = 1.0
    grid_spacing: int = 32
    search_radius_x: int = 25
    search_radius_y: int = 25
    min_search_radius: int = 6
    coarse_stride: int = 4
    coarse_buffer: int = 8
    min_coarse_valid_fraction: float = 0.01
    dx_prior: float = 0.0
    dy_prior: float = 0.0
    fill_window: int = 3
    rng_seed: int = 0
    progress: bool = False


def chip_sizes(p: Params):
    """Chip-size levels, ascending (src/types.jl:842-850)."""
    out = []
    cs = p.chip_size_base
    while cs <= p.chip_size_max:
        if cs >= p.chip_size_min:
            out.append(cs)
        cs *= 2
    return out


def chip_size_y(p: Params, chip_size_x: int) -> int:
    """Chip height for a width, forced even (src/types.jl:914-915); Julia rounds half to even."""
    return 2 * int(round(chip_size_x * p.chip_aspect / 2))


def measure_at(p: Params, level: int):
    """The measure of level `level` (1 = finest), last entry repeating (src/types.jl:891-892)."""
    return p.similarity[min(level, len(p.similarity)) - 1]


_SIMILARITY = {"zncc": ZNCC(), "ncc": NCC(), "coherence": Coherence()}
_QUANTIZE = {"uint8": QuantizeUInt8(), "none": NoQuantize()}
_PREPROCESS = {"highpass": Highpass, "wallis": Wallis, "none": NoPreprocess}
_SUBPIXEL = {"pyramid": PyramidRefine, "none": NoRefine}
_OUTLIERS = {"gardner": GardnerFilter, "none": NoOutlierFilter}


def _resolve(table, x, kw):
    if x in table:
        return table[x]
    valid = ", ".join(f":{k}" for k in sorted(table))
    raise ValueError(f"`{kw} = :{x}` is not recognised. Valid options are {valid}.")


def _check_chip_size(name, cs):
    if cs <= 0:
        raise ValueError(f"`{name}` must be positive, got {cs}")
    if cs % 4:
        raise ValueError(f"`{name}` must be a multiple of 4, got {cs}. Chip sizes are halved at "
                         "each chip-size level and need an even half-extent in both directions.")
    return int(cs)


def _pair(x):
    if isinstance(x, (tuple, list)):
        if len(x) != 2:
            raise ValueError(f"expected 1 or 2 values, got {len(x)}")
        return int(x[0]), int(x[1])
    return int(x), int(x)


_NOKW = object()


def params(*, similarity="zncc", preprocess="highpass", quantize="uint8", subpixel="pyramid",
           filter_width=_NOKW, upsampling=_NOKW, chip_size=32, chip_size_min=_NOKW,
           chip_size_max=_NOKW, chip_aspect=1.0, grid_spacing=_NOKW, search_radius=25,
           search_radius_x=_NOKW, search_radius_y=_NOKW, min_search_radius=6, dx_prior=0.0,
           dy_prior=0.0, coarse_stride=4, coarse_buffer=8, min_coarse_valid_fraction=0.01,
           outliers="gardner", rotation=None, outlier_window=_NOKW, outlier_iterations=_NOKW,
           min_agree_fraction=_NOKW, agree_tolerance=_NOKW, mad_scale=_NOKW, fill_window=3,
           threaded=False, progress=False, rng_seed=0) -> Params:
    """Resolve and validate keywords into a `Params` (src/params.jl:306-392)."""
    if isinstance(similarity, tuple):
        if not similarity:
            raise ValueError("`similarity` cannot be an empty tuple; name at least one measure.")
        sim = tuple(_resolve(_SIMILARITY, s, "similarity") if isinstance(s, str) else s
                    for s in similarity)
    else:
        sim = (_resolve(_SIMILARITY, similarity, "similarity")
               if isinstance(similarity, str) else similarity,)

    if isinstance(preprocess, str):
        T = _resolve(_PREPROCESS, preprocess, "preprocess")
        pre = T() if (T is NoPreprocess or filter_width is _NOKW) else T(width=int(filter_width))
    else:
        pre = preprocess
    quant = _resolve(_QUANTIZE, quantize, "quantize") if isinstance(quantize, str) else quantize
    if isinstance(subpixel, str):
        T = _resolve(_SUBPIXEL, subpixel, "subpixel")
        sub = NoRefine() if T is NoRefine else (
            T() if upsampling is _NOKW else T(upsampling=int(upsampling)))
    else:
        sub = subpixel

    okw = dict(window=outlier_window, iterations=outlier_iterations,
               min_agree_fraction=min_agree_fraction, agree_tolerance=agree_tolerance,
               mad_scale=mad_scale)
    given = {k: v for k, v in okw.items() if v is not _NOKW}
    if isinstance(outliers, str):
        T = _resolve(_OUTLIERS, outliers, "outliers")
        if T is NoOutlierFilter:
            if given:
                raise ValueError(f"`outliers` was given `:{outliers}`, which takes no parameters, "
                                 f"so {', '.join(f'`{k}`' for k in given)} cannot also apply.")
            out = NoOutlierFilter()
        else:
            out = T(**given)
    else:
        if given:
            raise ValueError(f"`outliers` was given a {type(outliers).__name__} instance, which "
                             "already carries its own parameters, so "
                             f"{', '.join(f'`{k}`' for k in given)} cannot also apply.")
        out = outliers
    rot = _rotation(rotation)

    base = _check_chip_size("chip_size", chip_size)
    cmin = base if chip_size_min is _NOKW else _check_chip_size("chip_size_min", chip_size_min)
    cmax = 4 * base if chip_size_max is _NOKW else _check_chip_size("chip_size_max", chip_size_max)
    if cmin > cmax:
        raise ValueError(f"`chip_size_min` ({cmin}) must be <= `chip_size_max` ({cmax})")
    if base > cmin:
        raise ValueError(f"`chip_size` ({base}) must be <= `chip_size_min` ({cmin}). `chip_size` "
                         "is the finest chip-size level; coarser levels are its powers-of-two "
                         "multiples.")
    if cmax % base:
        raise ValueError(f"`chip_size_max` ({cmax}) must be a power-of-two multiple of "
                         f"`chip_size` ({base}), because chip-size levels double at each step.")
    ratio = cmax // base
    if ratio & (ratio - 1):
        raise ValueError(f"`chip_size_max` ({cmax}) must be a power-of-two multiple of "
                         f"`chip_size` ({base}), got a ratio of {ratio}.")
    if grid_spacing is _NOKW:
        spacing = base
    else:
        if not grid_spacing > 0:
            raise ValueError(f"`grid_spacing` must be positive, got {grid_spacing}")
        spacing = int(grid_spacing)
    rx0, ry0 = _pair(search_radius)
    rx = rx0 if search_radius_x is _NOKW else int(search_radius_x)
    ry = ry0 if search_radius_y is _NOKW else int(search_radius_y)
    if rx < 0:
        raise ValueError(f"`search_radius_x` must be >= 0, got {rx}")
    if ry < 0:
        raise ValueError(f"`search_radius_y` must be >= 0, got {ry}")
    if not (rx > 0 or ry > 0):
        raise ValueError("`search_radius` is zero in both axes, so no pixel can be searched.")
    if not chip_aspect > 0:
        raise ValueError(f"`chip_aspect` must be positive, got {chip_aspect}")
    if not coarse_stride > 0:
        raise ValueError(f"`coarse_stride` must be positive, got {coarse_stride}")
    if not (0 <= min_coarse_valid_fraction <= 1):
        raise ValueError("`min_coarse_valid_fraction` must be in [0, 1], got "
                         f"{min_coarse_valid_fraction}")
    if fill_window < 1:
        raise ValueError(f"`fill_window` must be >= 1, got {fill_window}")
    if fill_window % 2 == 0:
        raise ValueError(f"`fill_window` must be odd so the window has a centre pixel, "
                         f"got {fill_window}")
    return Params(similarity=sim, preprocess=pre, quantize=quant, subpixel=sub, outliers=out,
                  threaded=bool(threaded), rotation=rot, chip_size_base=base,
                  chip_size_min=cmin, chip_size_max=cmax, chip_aspect=float(chip_aspect),
                  grid_spacing=spacing, search_radius_x=rx, search_radius_y=ry,
                  min_search_radius=int(min_search_radius), coarse_stride=int(coarse_stride),
                  coarse_buffer=int(coarse_buffer),
                  min_coarse_valid_fraction=float(min_coarse_valid_fraction),
                  dx_prior=float(dx_prior), dy_prior=float(dy_prior),
                  fill_window=int(fill_window), rng_seed=int(rng_seed), progress=bool(progress))
