"""UInt8 surfaces of 66..128 rows or columns (radii 33..64, beyond k_corr_tc2's 64 x 64, on
k_corr_tc's 128-row products): every result bit-identical to the oracle for power-of-two chip
areas, and to the CUDA-core path (tensor cores off) for any chip, including passes that mix
them with smaller surfaces, points in the zero padding, priors and masks, and the multichip
search."""

import numpy as np
import pytest

from conftest import fields
from test_gpu_parity import assert_identical, run_both

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("chip,radius,spacing,up", [
    (32, 33, 24, 64), (32, 47, 30, 16), (16, 44, 20, 64), (64, 40, 40, 64), (32, 64, 40, 1),
    (16, 35, 16, 8), (32, 48, 36, 2)])
def test_split_surfaces_bit_identical(ar, O, gpu_lib, chip, radius, spacing, up):
    ref, sec = ar.synthetic.shifted_pair(360, (6.4, -3.7), seed=chip + radius, dtype=np.uint8)
    pts = ar.gridpoints(ref.shape, spacing, chip_size=chip, search_radius=radius)
    g, w = run_both(ar, O, ref, sec, pts, up=up)
    assert w[3].any()
    assert_identical(g, w)


def _direct(ar, pair, pts, p, sub):
    ctx = ar._lib.Context(0)
    ctx.set_option(ar._lib.AR_OPT_TENSOR_CORES, 0)
    d = ar.track(pair, pts, p, subpixel=sub, ctx=ctx)
    ctx.close()
    return d


def test_split_mixed_radii_padding_priors_masks(ar, O, gpu_lib):
    """One pass mixing whole and split surfaces, non-square radii, non-power-of-two chips,
    points in the zero padding, fractional priors and masks: identical to the CUDA-core path,
    and to the oracle for power-of-two chip areas."""
    rng = np.random.default_rng(7)
    ref, sec = ar.synthetic.shifted_pair(300, (5.25, 2.5), seed=4, dtype=np.uint8)
    n = 500
    pts = ar.pointset(rng.uniform(-5, 306, n), rng.uniform(-5, 306, n),
                      chip_size=rng.choice([16, 20, 32], n), chip_size_y=rng.choice([16, 24, 32], n),
                      search_radius_x=rng.integers(1, 60, n), search_radius_y=rng.integers(1, 60, n),
                      dx_prior=np.round(rng.normal(0, 4, n)), dy_prior=rng.normal(0, 3, n))
    rv = np.ones(ref.shape, bool)
    rv[100:140, 30:90] = False
    sv = np.ones(ref.shape, bool)
    sv[:, 240:] = False
    pair = ar.ImagePair(ref, sec, rv, sv)
    p = ar.params(preprocess="none", quantize="none", upsampling=16)
    sub = ar.PyramidRefine(16)
    got = ar.track(pair, pts, p, subpixel=sub)
    direct = _direct(ar, pair, pts, p, sub)
    for name in ("dx", "dy", "correlation"):
        a, b = getattr(got, name), getattr(direct, name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
    assert np.array_equal(got.searched, direct.searched)
    big = (2 * pts.radius_x > 64) | (2 * pts.radius_y > 64)
    assert big.sum() > 100 and (~big).sum() > 100
    want = O.track(ref, sec, fields(pts), upsampling=16, reference_valid=rv, secondary_valid=sv)
    area = (2 * (pts.chip_size_x // 2)) * (2 * (pts.chip_size_y // 2))
    p2 = ((area & (area - 1)) == 0).ravel(order="F")
    g = tuple(a.ravel(order="F")[p2] for a in (got.dx, got.dy, got.correlation, got.searched))
    assert_identical(g, tuple(a[p2] for a in want))


def test_split_multichip(ar, O, gpu_lib):
    """The multichip search with radius 40 at chips 32/64 (split at every level) against the
    oracle."""
    from test_gpu_multichip import check_identical
    from test_oracle_multichip import mc_params
    ref, sec = ar.synthetic.shifted_pair(420, (9.5, -12.25), seed=3, dtype=np.uint8)
    grid = ar.gridpoints(ref.shape, 24, chip_size=64, search_radius=40)
    p = ar.params(chip_size=32, chip_size_max=64, search_radius=40, preprocess="none",
                  quantize="none")
    got = ar.correlate_multichip(ar.ImagePair(ref, sec), grid, p)
    want = O.multichip(ref, sec, fields(grid), mc_params(ar, p))
    check_identical(got, want)
