"""The oracle's multi-chip-size search and outlier filter against the reference's own tests
(test/multichip.jl, test/outliers.jl), restated."""

import numpy as np
import pytest

from conftest import fields


def mc_params(ar, p):
    """The oracle's parameter dict for a Params."""
    o = p.outliers
    g = isinstance(o, ar.GardnerFilter)
    return dict(chip_base=p.chip_size_base, chip_min=p.chip_size_min, chip_max=p.chip_size_max,
                aspect=p.chip_aspect, min_radius=p.min_search_radius, stride=p.coarse_stride,
                buffer=p.coarse_buffer, min_frac=p.min_coarse_valid_fraction,
                up=ar.upsampling(p.subpixel),
                measure=1 if type(p.similarity[0]).__name__ == "NCC" else 0,
                outliers=1 if g else 0,
                window=o.window if g else 5, iterations=o.iterations if g else 3,
                min_agree_fraction=o.min_agree_fraction if g else 0.32,
                agree_tolerance=o.agree_tolerance if g else 0.2,
                mad_scale=o.mad_scale if g else 4.0, fill_window=p.fill_window,
                level_measures=[1 if type(m).__name__ == "NCC" else 0 for m in p.similarity]
                if len(p.similarity) > 1 else [])


def coherent_field(n, outliers=()):
    i, j = np.meshgrid(np.arange(1, n + 1), np.arange(1, n + 1), indexing="ij")
    dx = (np.float32(3.0) + np.float32(0.05) * i.astype(np.float32)).astype(np.float32)
    dy = (np.float32(-2.0) - np.float32(0.05) * j.astype(np.float32)).astype(np.float32)
    for (a, b, vx, vy) in outliers:
        dx[a - 1, b - 1] = vx
        dy[a - 1, b - 1] = vy
    return dx, dy


def test_coherent_field_survives(O):
    n = 20
    dx, dy = coherent_field(n)
    r = np.full((n, n), 25)
    keep = O.reject_outliers(dx, dy, r, r, np.ones((n, n), bool), 64)
    assert keep[3:n - 3, 3:n - 3].all()
    assert keep.mean() > 0.6


def test_isolated_outliers_rejected(O):
    n = 20
    spikes = ((6, 6, 20.0, 20.0), (12, 9, -22.0, 18.0), (15, 15, 24.0, -24.0))
    dx, dy = coherent_field(n, spikes)
    r = np.full((n, n), 25)
    keep = O.reject_outliers(dx, dy, r, r, np.ones((n, n), bool), 64)
    for (i, j, _, _) in spikes:
        assert not keep[i - 1, j - 1]
    assert keep[2, 2] and keep[9, 9]


def test_rejection_monotone_and_invalid_stay_invalid(O):
    n = 16
    dx, dy = coherent_field(n, ((8, 8, 30.0, 30.0),))
    r = np.full((n, n), 25)
    prev = np.ones((n, n), bool)
    for it in range(1, 5):
        keep = O.reject_outliers(dx, dy, r, r, np.ones((n, n), bool), 64, iterations=it)
        assert np.all(~keep | prev)
        prev = keep
    valid = np.ones((n, n), bool)
    valid[4, 4] = False
    rx = r.copy()
    rx[2, 2] = 0
    keep = O.reject_outliers(dx, dy, rx, r, valid, 64)
    assert not keep[4, 4] and not keep[2, 2]


@pytest.mark.parametrize("shift", [(0, 0), (5, -3)])
def test_exact_recovery_through_the_pyramid(ar, O, shift):
    sx, sy = shift
    ref, sec = ar.synthetic.shifted_pair(512, shift)
    grid = ar.gridpoints((512, 512), 32, chip_size=32, search_radius=25)
    p = ar.params(chip_size=32, chip_size_max=128)
    dx, dy, c, cs, it = O.multichip(ref, sec, fields(grid), mc_params(ar, p))
    assert np.isfinite(dx).all()
    assert abs(np.median(-dx) - sx) <= 0.05 and abs(np.median(-dy) - sy) <= 0.05
    assert np.all(cs == 32)


def banded_pair(ar, n, shift, band):
    ref, sec = ar.synthetic.shifted_pair(n, shift)
    ref = ref.copy(); sec = sec.copy()
    ref[band] = 0.5
    sec[band] = 0.5
    return ref, sec


def test_coarser_levels_recover_what_finer_ones_cannot(ar, O):
    n = 512
    ref, sec = banded_pair(ar, n, (6, -4), slice(199, 290))
    grid = ar.gridpoints((n, n), 32, chip_size=32, search_radius=25)
    counts = []
    for cmax in (32, 64, 128):
        p = ar.params(chip_size=32, chip_size_max=cmax)
        dx, dy, c, cs, it = O.multichip(ref, sec, fields(grid), mc_params(ar, p))
        counts.append(int(np.isfinite(dx).sum()))
        used = set(np.unique(cs[cs > 0]).tolist())
        assert used <= {32, 64, 128} and 32 in used
        if cmax >= 64:
            assert 64 in used
        assert np.array_equal(cs == 0, np.isnan(dx))
    assert counts[0] < counts[1] < counts[2] < len(grid)
