"""The tensor-core correlation (k_corr_tc) against the CUDA-core kernel on UInt8 passes.

Both compute the exact integer numerator, the same box sums and the reference's FP64
normalisation, so every output must be bit-identical: dx, dy, correlation, searched, and the
full surfaces. The cases cover the track semantics the kernel re-implements: priors, padding at
image borders, masks, per-point radii and chip sizes, NCC, non-square surfaces and chip areas
that are not powers of two.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def both(ar, fn):
    ctx = ar._lib.default_context()
    try:
        ctx.set_option(ar._lib.AR_OPT_TENSOR_CORES, 1)
        a = fn(ctx)
        ctx.set_option(ar._lib.AR_OPT_TENSOR_CORES, 0)
        b = fn(ctx)
    finally:
        ctx.set_option(ar._lib.AR_OPT_TENSOR_CORES, 1)
    return a, b


def same_f(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def check_fields(a, b):
    for name in ("dx", "dy", "correlation"):
        assert same_f(getattr(a, name), getattr(b, name)), name
    assert np.array_equal(a.searched, b.searched)


CASES = [
    dict(chip=32, r=25, up=64, measure="zncc"),
    dict(chip=32, r=25, up=1, measure="ncc"),
    dict(chip=24, r=12, up=16, measure="zncc"),   # chip area 576: not a power of two
    dict(chip=16, r=(20, 8), up=8, measure="zncc"),
    dict(chip=32, r=(6, 31), up=32, measure="zncc"),
    dict(chip=32, r=(48, 20), up=16, measure="zncc"),   # 96 surface columns: M = 128
    dict(chip=16, r=(40, 40), up=8, measure="ncc"),
]


@pytest.mark.parametrize("case", CASES)
def test_track_identical(ar, gpu_lib, case):
    ref, sec = ar.synthetic.shifted_pair(384, (4.3, -2.6), seed=17, dtype=np.uint8)
    sv = np.ones(ref.shape, bool)
    sv[100:140, 200:260] = False
    rx, ry = case["r"] if isinstance(case["r"], tuple) else (case["r"], case["r"])
    rng = np.random.default_rng(5)
    n = 700
    x = rng.uniform(-10, 395, n)           # some windows leave the image: the padded path
    y = rng.uniform(-10, 395, n)
    pts = ar.pointset(x, y, chip_size=case["chip"], search_radius_x=rx, search_radius_y=ry,
                      dx_prior=np.round(rng.uniform(-3, 3, n)), dy_prior=rng.uniform(-2, 2, n))
    pair = ar.ImagePair(ref, sec, None, sv)
    p = ar.params(preprocess="none", quantize="none", similarity=case["measure"],
                  upsampling=case["up"] if case["up"] > 1 else 64,
                  subpixel="pyramid" if case["up"] > 1 else "none")
    a, b = both(ar, lambda ctx: ar.track(pair, pts, p, ctx=ctx))
    check_fields(a, b)
    assert np.count_nonzero(~np.isnan(a.dx)) > n // 3


@pytest.mark.parametrize("chip,r", [(64, 25), (128, 25), (96, 20), (128, 6)])
def test_track_large_chips_identical(ar, gpu_lib, chip, r):
    """Chips whose operand is built and multiplied in several chunks."""
    ref, sec = ar.synthetic.shifted_pair(640, (-5.3, 3.7), seed=29, dtype=np.uint8)
    rng = np.random.default_rng(chip + r)
    n = 300
    pts = ar.pointset(rng.uniform(60, 580, n), rng.uniform(60, 580, n), chip_size=chip,
                      search_radius=r, dy_prior=np.round(rng.uniform(-2, 2, n)))
    pair = ar.ImagePair(ref, sec)
    p = ar.params(preprocess="none", quantize="none", upsampling=16)
    a, b = both(ar, lambda ctx: ar.track(pair, pts, p, ctx=ctx))
    check_fields(a, b)
    assert np.count_nonzero(~np.isnan(a.dx)) > n // 2


def test_track_mixed_geometry(ar, gpu_lib):
    """Per-point radii (including 0: not searchable) and chip sizes in one pass."""
    ref, sec = ar.synthetic.shifted_pair(320, (-3.2, 5.4), seed=23, dtype=np.uint8)
    rng = np.random.default_rng(9)
    n = 500
    pts = ar.pointset(rng.uniform(40, 280, n), rng.uniform(40, 280, n),
                      chip_size=rng.choice([8, 16, 24, 32], n),
                      search_radius_x=rng.integers(0, 31, n), search_radius_y=rng.integers(0, 31, n))
    pair = ar.ImagePair(ref, sec)
    p = ar.params(preprocess="none", quantize="none")
    a, b = both(ar, lambda ctx: ar.track(pair, pts, p, ctx=ctx))
    check_fields(a, b)


def test_surfaces_identical(ar, gpu_lib):
    rng = np.random.default_rng(12)
    for (ch, cw, rx, ry) in [(32, 32, 25, 25), (24, 16, 10, 30), (32, 32, 32, 3)]:
        search = rng.integers(0, 256, (ch + 2 * ry - 1, cw + 2 * rx - 1), dtype=np.uint8)
        chip = rng.integers(0, 256, (ch, cw), dtype=np.uint8)
        chip[3:7, 5] = 0  # not constant rows
        for measure in (ar.ZNCC(), ar.NCC()):
            (sa, da), (sb, db) = both(
                ar, lambda ctx: ar.correlate(search, chip, (rx, ry), measure, ctx=ctx))
            assert da == db
            assert same_f(sa, sb)


def test_default_pipeline_identical(ar, gpu_lib):
    """The multichip pipeline (coarse NoRefine passes, fine passes, levels) with and without
    the tensor-core kernel."""
    a, b, valid, _ = ar.synthetic.scale_u16_pair(640, seed=4)
    p = ar.params(grid_spacing=8)
    grid = ar.build_grid(a.shape, p)

    def run(ctx):
        prep = ar.prepare(ar.ImagePair(a, b, None, valid), p, ctx)
        return ar.correlate_multichip(prep, grid, p, ctx)

    ra, rb = both(ar, run)
    for name in ("dx", "dy", "correlation"):
        assert same_f(getattr(ra, name), getattr(rb, name)), name
    assert np.array_equal(ra.chip_size, rb.chip_size)
    assert np.array_equal(ra.interpolated, rb.interpolated)
