"""Rotation search (src/track.jl:313-409, src/types.jl:529-577) on the CPU: the host-side
method objects and keyword resolution, the oracle's chip rotation against an independent
restatement, and the reference's behavioural tests (test/firstguess.jl:104-330) run on the
oracle. The GPU path is checked against the oracle in test_gpu_rotation.py."""

import ctypes
import math

import numpy as np
import pytest

from conftest import fields


# ---------------------------------------------------------------------------------------------
# Method objects and keywords (test/firstguess.jl:109-153)

def test_construction_and_the_off_case(ar):
    R, angles = ar.RotationSearch, ar.angles
    assert angles(R()) == (-3.0, 0.0, 3.0)
    assert angles(R((-1, 0, 1))) == (-1.0, 0.0, 1.0)
    with pytest.raises(ValueError):
        R(())
    with pytest.raises(ValueError):
        R((0.0, 3.0, 0.0))
    assert ar.params().rotation == ar.NoRotationSearch()
    assert ar.params(rotation=None).rotation == ar.NoRotationSearch()
    assert ar.params(rotation=False).rotation == ar.NoRotationSearch()
    assert angles(ar.params(rotation=True).rotation) == (-3.0, 0.0, 3.0)
    assert angles(ar.params(rotation=(-2, 0, 2)).rotation) == (-2.0, 0.0, 2.0)
    assert angles(ar.params(rotation=range(-6, 7, 3)).rotation) == (-6.0, -3.0, 0.0, 3.0, 6.0)
    assert angles(ar.params(rotation=np.array([-1.5, 1.5])).rotation) == (-1.5, 1.5)
    with pytest.raises(ValueError):
        ar.params(rotation="yes")
    with pytest.raises(TypeError):
        angles(ar.NoRotationSearch())


def test_about_shifts_the_window(ar):
    R, angles = ar.RotationSearch, ar.angles
    assert angles(R(about=8.0)) == (-11.0, -8.0, -5.0)
    assert angles(R((-1, 0, 1), about=-4.5)) == (3.5, 4.5, 5.5)
    assert angles(R()) == angles(R(about=0.0))
    for bad in (dict(about=math.nan), dict(angles=(-3, 0, 3), about=math.inf),
                dict(angles=(math.nan, 0.0, 3.0)), dict(angles=(-math.inf, 0.0, 3.0))):
        with pytest.raises(ValueError):
            R(**bad)
    # An unfittable scene rotation (`nothing` in the reference, None here) is a type error.
    with pytest.raises(TypeError):
        R(about=None)
    assert angles(R((0.0,), about=-8.0)) == (8.0,)


def test_device_angle_limit(ar):
    ar.RotationSearch(tuple(range(64)))
    with pytest.raises(ValueError):
        ar.RotationSearch(tuple(range(65)))


def test_multichip_params_carry_the_angles(ar):
    prm = ar.multichip_params(ar.params(rotation=ar.RotationSearch((-2.0, 1.0), about=0.5)))
    assert prm.rotation_count == 2
    got = np.ctypeslib.as_array((ctypes.c_double * 2).from_address(prm.rotation_angles))
    assert tuple(got) == (-2.5, 0.5)
    assert ar.multichip_params(ar.params()).rotation_count == 0


# ---------------------------------------------------------------------------------------------
# The oracle's chip rotation (src/track.jl:377-409)

def _rotate_py(c, deg):
    """A second, loop-by-loop restatement of _rotate_chip."""
    ch, cw = c.shape
    r = deg * (math.pi / 180.0)
    s, co = math.sin(r), math.cos(r)
    yc, xc = (ch + 1) / 2, (cw + 1) / 2
    out = np.zeros((ch, cw), np.float32)
    for j in range(1, cw + 1):
        for i in range(1, ch + 1):
            dy, dx = i - yc, j - xc
            sy = yc + co * dy + s * dx
            sx = xc - s * dy + co * dx
            i0, j0 = math.floor(sy), math.floor(sx)
            if i0 < 1 or j0 < 1 or i0 + 1 > ch or j0 + 1 > cw:
                continue
            fy, fx = sy - i0, sx - j0
            v00, v10 = float(c[i0 - 1, j0 - 1]), float(c[i0, j0 - 1])
            v01, v11 = float(c[i0 - 1, j0]), float(c[i0, j0])
            out[i - 1, j - 1] = np.float32((1 - fy) * ((1 - fx) * v00 + fx * v01) +
                                           fy * ((1 - fx) * v10 + fx * v11))
    return out


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.float32, np.int16])
def test_oracle_rotate_chip_matches_restatement(O, dtype):
    rng = np.random.default_rng(4)
    if np.dtype(dtype).kind == "f":
        chip = rng.standard_normal((14, 10)).astype(dtype)
    else:
        info = np.iinfo(dtype)
        chip = rng.integers(max(info.min, -3000), min(info.max, 3000) + 1, (14, 10)).astype(dtype)
    chip = np.asfortranarray(chip)
    for deg in (-3.0, 3.0, 0.5, -7.25, 45.0, 90.0, 180.0):
        assert np.array_equal(O.rotate_chip(chip, deg), _rotate_py(chip, deg)), deg


def test_rotate_chip_geometry(O):
    c = np.asfortranarray(np.arange(1, 26, dtype=np.float64).reshape(5, 5))
    # A quarter turn of an odd square chip moves every interior sample onto another sample.
    q = O.rotate_chip(c, 90.0)
    assert np.allclose(q[1:4, 1:4], np.rot90(c, 1)[1:4, 1:4], atol=1e-5) or \
        np.allclose(q[1:4, 1:4], np.rot90(c, -1)[1:4, 1:4], atol=1e-5)
    # The centre is fixed by every rotation.
    for deg in (-3.0, 17.0, 90.0):
        assert abs(O.rotate_chip(c, deg)[2, 2] - c[2, 2]) < 1e-4


# ---------------------------------------------------------------------------------------------
# The reference's behavioural tests, on the oracle

def _one_point(ar, ci, cj, cs, R):
    return ar.pointset([float(cj)], [float(ci)], chip_size=cs, search_radius=R)


def test_counter_rotation_recovers_correlation(ar, O):
    """test/firstguess.jl:244-287: a chip from the rotated secondary, turned back, correlates
    better than turned the wrong way at every chip size, and better than unturned once the
    chip is large enough for its corners to have moved."""
    n, motion, R = 512, 8.0, 4
    a = ar.synthetic.synthetic_texture((n, n), seed=3)
    b = ar.synthetic.rotate_bilinear(a, motion)

    def peak(cs, ang):
        pts = _one_point(ar, 257, 257, cs, R)
        _, _, c, s = O.track(a, b, fields(pts), upsampling=1, angles=(ang,))
        assert s[0]
        return float(c[0])

    for cs in (32, 64, 128):
        back, unrot, wrong = peak(cs, -motion), peak(cs, 0.0), peak(cs, motion)
        assert back > wrong, cs
        if cs >= 64:
            assert back > unrot, cs
    assert ar.angles(ar.RotationSearch((0.0,), about=-motion)) == (motion,)


def test_single_zero_angle_is_the_unrotated_path(ar, O):
    """test/firstguess.jl:289-307 on the oracle: RotationSearch((0.0,)) correlates the chip
    itself, so every output equals the plain pass."""
    ref, sec = ar.synthetic.shifted_pair(160, (4, -3), seed=2, dtype=np.float32)
    pts = ar.gridpoints(ref.shape, 16, chip_size=32, search_radius=10)
    off = O.track(ref, sec, fields(pts), upsampling=16)
    one = O.track(ref, sec, fields(pts), upsampling=16, angles=(0.0,))
    for x, y in zip(off, one):
        assert np.array_equal(x, y, equal_nan=x.dtype.kind == "f")


def test_best_angle_is_kept(ar, O):
    """The kept surface is the angle with the strictly highest peak: the search's correlation is
    the maximum of the single-angle correlations."""
    n = 256
    a = ar.synthetic.synthetic_texture((n, n), seed=8)
    b = ar.synthetic.rotate_bilinear(a, 4.0)
    pts = ar.gridpoints(a.shape, 24, chip_size=48, search_radius=6)
    angs = (-4.0, 0.0, 4.0)
    _, _, c3, _ = O.track(a, b, fields(pts), upsampling=1, angles=angs)
    singles = np.stack([O.track(a, b, fields(pts), upsampling=1, angles=(g,))[2] for g in angs])
    m = ~np.isnan(c3)
    assert m.sum() > 20
    assert np.array_equal(c3[m], np.nanmax(singles[:, m], axis=0))
    # A subset of the angles never finds a higher peak.
    _, _, c2, _ = O.track(a, b, fields(pts), upsampling=1, angles=(-4.0, 0.0))
    assert np.all(c2[m] <= c3[m])


def test_every_angle_degenerate_is_no_measurement(ar, O):
    ref = np.zeros((120, 120), np.uint8)
    pts = ar.gridpoints(ref.shape, 30, chip_size=16, search_radius=5)
    dx, dy, c, s = O.track(ref, ref, fields(pts), upsampling=16, angles=(-3.0, 0.0, 3.0))
    assert s.all() and np.isnan(dx).all() and np.isnan(c).all()


def test_turned_flat_chip_is_not_degenerate(ar, O):
    """A flat nonzero chip is degenerate unturned, but a turned copy has zero corners (samples
    from outside the chip), so it has texture and the search measures it."""
    ref = np.full((120, 120), 7, np.uint8)
    pts = ar.gridpoints(ref.shape, 30, chip_size=16, search_radius=5)
    dx0, _, _, s0 = O.track(ref, ref, fields(pts), upsampling=16, angles=(0.0,))
    assert s0.all() and np.isnan(dx0).all()
    dx, _, c, s = O.track(ref, ref, fields(pts), upsampling=16, angles=(-3.0, 0.0, 3.0))
    assert s.all() and np.isfinite(dx).all() and np.isfinite(c).all()


def test_rotation_search_recovers_correlation_lost_to_rotation(ar, O):
    """test/firstguess.jl:309-330: a scene rotated by 3 degrees correlates better with the
    search than without it (median correlation at least 5% higher)."""
    n = 256
    a = ar.synthetic.synthetic_texture((n, n), seed=5)
    b = ar.synthetic.rotate_bilinear(a, 3.0)
    pa, _ = O.prepare(a, preprocess="highpass", quantize="none")
    pb, _ = O.prepare(b, preprocess="highpass", quantize="none")
    p = ar.params(chip_size=32, chip_size_max=32, search_radius=8, quantize="none",
                  outliers="none")
    grid = ar.build_grid(a.shape, p)
    prm = dict(chip_base=32, chip_min=32, chip_max=32, aspect=1.0, min_radius=6, stride=4,
               buffer=8, min_frac=0.01, up=64, measure=0, outliers=0, window=5, iterations=3,
               min_agree_fraction=8 / 25, agree_tolerance=0.2, mad_scale=4.0, fill_window=3)
    g = fields(grid)
    plain = O.multichip(pa, pb, g, prm)[2]
    rot = O.multichip(pa, pb, g, prm, angles=(-3.0, 0.0, 3.0))[2]
    cp = np.median(plain[~np.isnan(plain)])
    cr = np.median(rot[~np.isnan(rot)])
    assert cr > 1.05 * cp, (cp, cr)
