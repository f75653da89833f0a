"""The multi-chip-size search on the GPU (ar_multichip) against the oracle, and the public
lifecycle (autorift, init / reinit_ / autorift_, src/api.jl:66-274).

UInt8 imagery with power-of-two chip areas tracks bit-identically (test_gpu_parity.py), and
every grid pass (Gardner stages, dilation, nearest resampling, hole filling, merge) repeats
the reference's Float32/Float64 operations, so the whole MultichipResult must be identical.
"""

import numpy as np
import pytest

from conftest import fields
from test_oracle_multichip import banded_pair, mc_params

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(a, b) if a.dtype.kind != "f" else bool(
        np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def check_identical(got, want):
    names = ("dx", "dy", "correlation", "chip_size", "interpolated")
    for g, w, n in zip((got.dx, got.dy, got.correlation, got.chip_size, got.interpolated), want, names):
        assert g.shape == w.shape, n
        assert same(g, w), f"{n}: {np.count_nonzero(~((g == w) | (np.isnan(g) & np.isnan(w))) if g.dtype.kind == 'f' else g != w)} differ"


def u16_scene(ar, n=640, seed=5, amp=8.0):
    a, b, valid, _ = ar.synthetic.scale_u16_pair(n, seed=seed, max_amp=amp)
    return a, b, valid


def test_default_pipeline_identical_to_oracle(ar, O, gpu_lib):
    a, b, sv = u16_scene(ar)
    p = ar.params(grid_spacing=8)
    prep = ar.prepare(ar.ImagePair(a, b, None, sv), p)
    grid = ar.build_grid(a.shape, p)
    got = ar.correlate_multichip(prep, grid, p)
    wr, wrm = O.prepare(a, None, "highpass", 5)
    ws, wsm = O.prepare(b, sv, "highpass", 5)
    want = O.multichip(wr, ws, fields(grid), mc_params(ar, p), wrm, wsm)
    check_identical(got, want)
    assert np.isfinite(got.dx).mean() > 0.8


@pytest.mark.parametrize("kind", ["int16_highpass", "float32_wallis"])
def test_other_input_types_default_pipeline(ar, O, gpu_lib, kind):
    """Int16 imagery (highpass) and Float32 imagery (Wallis), quantised to UInt8, through the
    multichip search: the GPU-prepared pair agrees with the oracle's preparation to within the
    quantiser's rounding-boundary allowance, and the multichip search on that prepared pair is
    identical to the oracle's."""
    a, b, sv = u16_scene(ar, n=512, seed=13)
    if kind == "int16_highpass":
        a = (a.astype(np.int32) - 32768).astype(np.int16)
        b = (b.astype(np.int32) - 32768).astype(np.int16)
        p = ar.params(grid_spacing=8)
        pre = "highpass"
    else:
        a = a.astype(np.float32) / 65535
        b = b.astype(np.float32) / 65535
        p = ar.params(grid_spacing=8, preprocess="wallis")
        pre = "wallis"
    prep = ar.prepare(ar.ImagePair(a, b, None, sv), p)
    ref, sec, rv, svv = prep.download()
    assert ref.dtype == np.uint8
    allow = 2 if kind == "int16_highpass" else a.size // 1000
    for img, mask, g, gm in ((a, None, ref, rv), (b, sv, sec, svv)):
        w, wm = O.prepare(img, mask, pre, 5)
        assert np.array_equal(gm, wm)
        d = np.abs(g.astype(np.int32) - w.astype(np.int32))
        assert d.max() <= 1 and np.count_nonzero(d) <= allow
    grid = ar.build_grid(a.shape, p)
    got = ar.correlate_multichip(prep, grid, p)
    want = O.multichip(ref, sec, fields(grid), mc_params(ar, p), rv, svv)
    check_identical(got, want)
    assert np.isfinite(got.dx).mean() > 0.8


def test_multilevel_banded_scene(ar, O, gpu_lib):
    ref, sec = banded_pair(ar, 512, (6, -4), slice(199, 290))
    ref8 = np.round(ref * 255).astype(np.uint8)
    sec8 = np.round(sec * 255).astype(np.uint8)
    grid = ar.gridpoints((512, 512), 16, chip_size=32, search_radius=25)
    for cmax in (64, 128):
        p = ar.params(chip_size=32, chip_size_max=cmax, preprocess="none", quantize="none")
        got = ar.correlate_multichip(ar.ImagePair(ref8, sec8), grid, p)
        want = O.multichip(ref8, sec8, fields(grid), mc_params(ar, p))
        check_identical(got, want)
        assert set(np.unique(got.chip_size[got.chip_size > 0]).tolist()) >= {32, 64}


def test_no_outlier_filter_and_ncc(ar, O, gpu_lib):
    a, b, sv = u16_scene(ar, n=640, seed=9)
    for kw in (dict(outliers="none"), dict(similarity="ncc"), dict(fill_window=5, mad_scale=3.0)):
        p = ar.params(grid_spacing=16, **kw)
        prep = ar.prepare(ar.ImagePair(a, b, None, sv), p)
        grid = ar.build_grid(a.shape, p)
        got = ar.correlate_multichip(prep, grid, p)
        wr, wrm = O.prepare(a, None, "highpass", 5)
        ws, wsm = O.prepare(b, sv, "highpass", 5)
        prm = mc_params(ar, p)
        prm["measure"] = 1 if kw.get("similarity") == "ncc" else 0
        want = O.multichip(wr, ws, fields(grid), prm, wrm, wsm)
        check_identical(got, want)


def test_exact_recovery_and_lifecycle(ar, gpu_lib):
    ref, sec = ar.synthetic.shifted_pair(512, (5, -3), dtype=np.uint8)
    r = ar.autorift(ref, sec, chip_size=32, search_radius=25)
    assert abs(np.nanmedian(-r.dx) - 5) <= 0.05 and abs(np.nanmedian(-r.dy) + 3) <= 0.05
    assert np.array_equal(r.chip_size == 0, np.isnan(r.dx))
    cache = ar.init(ref, sec, chip_size=32, search_radius=25)
    r1 = ar.autorift_(cache)
    assert ar.autorift_(cache) is r1                      # idempotent until reinit_
    for x, y in zip((r.dx, r.dy, r.correlation, r.chip_size), (r1.dx, r1.dy, r1.correlation, r1.chip_size)):
        assert same(x, y)                                 # cache equals one-shot
    ref2, sec2 = ar.synthetic.shifted_pair(512, (-2, 4), seed=3, dtype=np.uint8)
    ar.reinit_(cache, reference=ref2, secondary=sec2)
    r2 = ar.autorift_(cache)
    assert abs(np.nanmedian(-r2.dx) + 2) <= 0.05 and abs(np.nanmedian(-r2.dy) - 4) <= 0.05
    fresh = ar.autorift(ref2, sec2, chip_size=32, search_radius=25)
    assert same(fresh.dx, r2.dx) and same(fresh.chip_size, r2.chip_size)
    with pytest.raises(ValueError, match="built for"):
        ar.reinit_(cache, reference=ref2[:100])


def test_scattered_points_run_one_scale(ar, gpu_lib):
    ref, sec = ar.synthetic.shifted_pair(300, (3, 0), dtype=np.uint8)
    pts = ar.pointset([100.0, 187.5, 220.25, 140.0], [150.0, 120.0, 200.75, 99.5], chip_size=32,
                      search_radius=25)
    d = ar.autorift(ref, sec, pts, preprocess="none", quantize="none")
    assert d.dx.shape == (4,) and np.all(np.abs(-d.dx - 3) <= 0.05)


def test_per_level_similarity(ar, O, gpu_lib):
    """A `similarity` tuple: level k uses its k-th measure, the last repeating (measure_at,
    src/types.jl:893-894) -- the coarse and fine passes of each level alike. The banded scene
    leaves points to the coarser levels."""
    ref, sec = banded_pair(ar, 512, (6, -4), slice(199, 290))
    ref8 = np.round(ref * 255).astype(np.uint8)
    sec8 = np.round(sec * 255).astype(np.uint8)
    grid = ar.gridpoints((512, 512), 16, chip_size=32, search_radius=25)
    for sim in (("zncc", "ncc"), ("ncc", "zncc", "ncc"), ("ncc", "zncc")):
        p = ar.params(chip_size=32, chip_size_max=128, preprocess="none", quantize="none",
                      similarity=sim)
        got = ar.correlate_multichip(ar.ImagePair(ref8, sec8), grid, p)
        want = O.multichip(ref8, sec8, fields(grid), mc_params(ar, p))
        check_identical(got, want)
        assert (got.chip_size > 32).any()  # the later levels ran
