"""Known-answer tests of the oracle, restated from test/correlate.jl, test/peak.jl and
test/track.jl: exact integer shifts, self-correlation, degenerate chips, tie-breaking, the
peak origin, pyrUp brightness, fractional shifts and the grid-pass semantics.
"""

import numpy as np
import pytest

from conftest import fields


def chip_and_window(img, centre, cs, r, shift=(0, 0), window_from=None):
    """test/utils.jl:294-306: the chip is cut `shift` away, the window stays put."""
    cy, cx = centre
    sy, sx = shift
    h = cs // 2
    src = img if window_from is None else window_from
    chip = img[cy - h + sy - 1:cy + h - 1 + sy, cx - h + sx - 1:cx + h - 1 + sx]
    window = src[cy - h - r - 1:cy + h + r - 2, cx - h - r - 1:cx + h + r - 2]
    return chip, window


def test_exact_integer_shifts(O, ar):
    img = ar.synthetic.synthetic_texture((300, 300), seed=7)
    cs, r = 32, 25
    for sx, sy in ((0, 0), (3, -2), (7, 11), (-13, 5), (24, -24), (-24, 24)):
        chip, win = chip_and_window(img, (150, 150), cs, r, shift=(sy, sx))
        s, _ = O.correlate(win, chip, r)
        i, j = O.peak_index(s)
        assert (j - r, i - r) == (sx, sy)
        assert s[i, j] > 0.999


def test_self_correlation_is_one(O, ar):
    img = ar.synthetic.synthetic_texture((120, 120), seed=3)
    cs, r = 32, 10
    chip, win = chip_and_window(img, (60, 60), cs, r)
    s, _ = O.correlate(win, chip, r)
    assert O.peak_index(s) == (r, r)
    assert abs(float(s[r, r]) - 1.0) <= 1e-5
    assert np.all(s >= -1.0001) and np.all(s <= 1.0001)


def test_degenerate_chip_gives_zero_surface(O):
    win = np.random.default_rng(0).random((51, 51)).astype(np.float32)
    s, deg = O.correlate(win, np.full((32, 32), 5.0, np.float32), 10)
    assert deg and np.all(s == 0)


def test_peak_tie_breaking(O):
    a = np.zeros((7, 7), np.float32); a[3, 1] = a[3, 5] = 1
    assert O.peak_index(a) == (3, 1)
    a = np.zeros((7, 7), np.float32); a[1, 3] = a[5, 3] = 1
    assert O.peak_index(a) == (1, 3)
    a = np.zeros((7, 7), np.float32); a[2:5, 2:5] = 1
    assert O.peak_index(a) == (2, 2)
    assert O.peak_index(np.full((7, 7), 0.25, np.float32)) == (0, 0)
    a = np.zeros((5, 5), np.float32); a[1, 1] = np.nan; a[3, 3] = 0.5
    assert O.peak_index(a) == (3, 3)
    assert O.peak_index(np.full((3, 3), np.nan, np.float32)) == (0, 0)


def test_peak_offset_origin(O):
    r = 25
    a = np.zeros((2 * r, 2 * r), np.float32); a[r, r] = 1
    assert O.subpixel_peak(a, r, 1) == (0.0, 0.0, 1.0)
    a = np.zeros((2 * r, 2 * r), np.float32); a[r + 3, r + 7] = 1
    assert O.subpixel_peak(a, r, 1)[:2] == (7.0, 3.0)


def test_pyrup_brightness_and_mass(O):
    out = O.pyrup(np.full((5, 5), 0.5, np.float32))
    assert out.shape == (10, 10) and np.allclose(out, 0.5, atol=1e-5)
    d = np.zeros((5, 5), np.float32); d[2, 2] = 1
    assert abs(float(O.pyrup(d).sum()) - 4.0) < 1e-4


def test_fractional_shift_within_a_tenth(O, ar):
    for dx, dy in ((0.25, -0.5), (1.75, 0.6), (-2.3, 1.1)):
        ref, sec = ar.synthetic.shifted_pair(200, (dx, dy), seed=11)
        pts = ar.pointset([100.0], [100.0], chip_size=32, search_radius=10)
        gdx, gdy, c, s = O.track(ref, sec, fields(pts), upsampling=32)
        assert abs(-gdx[0] - dx) <= 0.1 and abs(-gdy[0] - dy) <= 0.1


@pytest.mark.parametrize("shift", [(0, 0), (5, -3), (-7, 11), (20, 20)])
def test_grid_recovers_integer_shift(O, ar, shift):
    sx, sy = shift
    ref, sec = ar.synthetic.shifted_pair(400, shift)
    pts = ar.gridpoints((400, 400), 32, chip_size=32, search_radius=25)
    dx, dy, c, s = O.track(ref, sec, fields(pts), upsampling=1)
    assert s.all() and np.isfinite(dx).all()
    assert np.all(-dx == sx) and np.all(-dy == sy)
    assert np.median(c) > 0.9
    dx, dy, c, s = O.track(ref, sec, fields(pts), upsampling=64)
    assert np.all(np.abs(-dx - sx) <= 3 / 64) and np.all(np.abs(-dy - sy) <= 3 / 64)


def test_unsearched_and_degenerate_points(O, ar):
    ref, sec = ar.synthetic.shifted_pair(300, (0, 0))
    ref = ref.copy(); sec = sec.copy()
    ref[99:200, 99:200] = 0.5
    sec[99:200, 99:200] = 0.5
    pts = ar.gridpoints((300, 300), 32, chip_size=32, search_radius=25)
    pts.radius_x[1, 1] = 0
    pts.radius_y[1, 1] = 0
    dx, dy, c, s = O.track(ref, sec, fields(pts), upsampling=64)
    S = s.reshape(pts.shape, order="F")
    DX = dx.reshape(pts.shape, order="F")
    assert not S[1, 1] and np.isnan(DX[1, 1])
    flat = (pts.x >= 130) & (pts.x <= 170) & (pts.y >= 130) & (pts.y <= 170)
    assert flat.any()
    assert S[flat].all() and np.isnan(DX[flat]).all()


def test_prior_centres_the_search(O, ar):
    sx, sy = 18, -14
    ref, sec = ar.synthetic.shifted_pair(400, (sx, sy))
    pts = ar.gridpoints((400, 400), 32, chip_size=32, search_radius=8,
                        dx_prior=-float(sx), dy_prior=-float(sy))
    dx, dy, c, s = O.track(ref, sec, fields(pts), upsampling=64)
    assert abs(np.nanmedian(-dx) - sx) < 0.5 and abs(np.nanmedian(-dy) - sy) < 0.5


def test_padding_path_zero_fills(O, ar):
    """A scattered point near the edge pads with zeros and a false mask (src/track.jl:128-138)."""
    ref, sec = ar.synthetic.shifted_pair(200, (2, 1))
    pts = ar.pointset([20.0, 100.0, 185.25], [15.5, 100.0, 190.0], chip_size=32,
                      search_radius=10)
    dx, dy, c, s = O.track(ref, sec, fields(pts), upsampling=16)
    assert s.all()
    assert abs(-dx[1] - 2) <= 0.1 and abs(-dy[1] - 1) <= 0.1
