"""Host-side logic that needs no GPU: parameter resolution (src/params.jl), point sets
(src/points.jl), the pass geometry the library computes (src/track.jl:176-197) and the bench
line's roofline helpers."""

from pathlib import Path

import numpy as np
import pytest


def test_params_defaults(ar):
    p = ar.params()
    assert isinstance(p.similarity[0], ar.ZNCC)
    assert p.preprocess == ar.Highpass(5)
    assert p.quantize == ar.QuantizeUInt8()
    assert p.subpixel == ar.PyramidRefine(64)
    assert p.outliers == ar.GardnerFilter()
    assert (p.chip_size_base, p.chip_size_min, p.chip_size_max) == (32, 32, 128)
    assert p.grid_spacing == 32 and (p.search_radius_x, p.search_radius_y) == (25, 25)
    assert p.min_search_radius == 6 and p.coarse_stride == 4 and p.coarse_buffer == 8
    assert ar.chip_sizes(p) == [32, 64, 128]


def test_params_validation(ar):
    with pytest.raises(ValueError, match="multiple of 4"):
        ar.params(chip_size=30)
    with pytest.raises(ValueError, match="power of 2"):
        ar.params(upsampling=48)
    with pytest.raises(ValueError, match="power-of-two multiple"):
        ar.params(chip_size=32, chip_size_max=96)
    with pytest.raises(ValueError, match="zero in both axes"):
        ar.params(search_radius=0)
    with pytest.raises(ValueError, match="not recognised"):
        ar.params(preprocess="nope")
    with pytest.raises(ValueError, match="cannot also apply"):
        ar.params(outliers="none", mad_scale=3.0)
    with pytest.raises(ValueError, match="odd"):
        ar.params(fill_window=4)
    p = ar.params(subpixel="none", search_radius=(30, 12), grid_spacing=8)
    assert ar.upsampling(p.subpixel) == 1
    assert (p.search_radius_x, p.search_radius_y, p.grid_spacing) == (30, 12, 8)


def test_gridpoints_layout(ar):
    pts = ar.gridpoints((512, 512), 32, chip_size=32, search_radius=25)
    # margin = cld(32, 2) + 25 + 1 = 42: centres 43:32:470, i.e. 14 per axis. (The reference's
    # docstring example says 13x13; its code, which this follows, gives 14x14, and its test
    # (test/points.jl:77-93) only asserts a square grid.)
    assert pts.shape == (14, 14)
    assert pts.x[0, 0] == 43 and pts.y[0, 0] == 43
    assert pts.x[0, 0] == pts.x[1, 0] and pts.y[0, 0] == pts.y[0, 1]
    assert pts.x[0, 1] > pts.x[0, 0] and pts.y[1, 0] > pts.y[0, 0]
    from autorift_b200.points import inbounds
    assert all(inbounds(pts, i, (512, 512)) for i in range(len(pts)))
    assert ar.gridpoints_xy(np.arange(100.0, 201.0, 10.0), np.arange(50.0, 101.0, 10.0),
                            chip_size=16).shape == (6, 11)
    assert np.all(pts.x[:, 1] == 75) and np.all(pts.y[1, :] == 75)
    assert np.all(pts.chip_size_y == 32) and np.all(pts.radius_x == 25)
    flat = pts.flat("x")
    assert flat[0] == 43 and flat[1] == 43 and flat[14] == 75  # column-major order
    with pytest.raises(ValueError, match="no search center fits"):
        ar.gridpoints((50, 50), 8, chip_size=32, search_radius=25)


def test_pointset_fields_and_aspect(ar):
    pts = ar.pointset([10.0, 50.5, 200.0], [20.0, 60.0, 30.25], search_radius=25, chip_size=32)
    assert len(pts) == 3 and pts.x[1] == 50.5 and pts.radius_x[1] == 25
    pts = ar.pointset([1.0, 2.0], [1.0, 2.0], chip_size=[32, 36], chip_aspect=0.5)
    assert list(pts.chip_size_y) == [16, 18]
    with pytest.raises(ValueError, match="integer"):
        ar.pointset([1.0], [1.0], chip_size=32.5)


def test_sanitize_rules(ar):
    pts = ar.pointset([1.0, 2, 3, 4], [1.0, 2, 3, 4], search_radius_x=[0, 3, 10, 4],
                      search_radius_y=[5, 0, 2, 9])
    n = ar.sanitize(pts, 6)
    assert n == 2
    assert list(pts.radius_x) == [0, 0, 10, 6]
    assert list(pts.radius_y) == [0, 0, 6, 9]


def test_decimation_copies(ar):
    pts = ar.gridpoints((400, 400), 8, chip_size=32, search_radius=25)
    coarse = pts[3::4, 3::4]
    coarse.radius_x[:] = 0
    assert np.all(pts.radius_x == 25)


def test_per_level_similarity_params(ar):
    prm = ar.multichip_params(ar.params(similarity=("zncc", "ncc")))
    assert prm.level_measure_count == 2 and list(prm.level_measures)[:2] == [0, 1]
    assert ar.multichip_params(ar.params()).level_measure_count == 0
    assert ar.multichip_params(ar.params(similarity=("ncc",))).measure == 1
    with pytest.raises(ValueError):
        ar.multichip_params(ar.params(similarity=("zncc", "ncc", "zncc", "ncc")))
    with pytest.raises(ValueError):
        ar.multichip_params(ar.params(similarity=("zncc", "coherence")))


def test_bench_traffic_and_fine_pass_kernel():
    """The bench line's roofline takes the fine pass's kernel from the autotuner's table and
    that kernel's committed DRAM bytes per point (None for a kernel without a capture)."""
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench

    class FakeCtx:
        def __init__(self, table):
            self.table = table

        def tuned(self):
            return self.table

    fine = {"chip": [bench.CHIP, bench.CHIP], "surface": [2 * bench.RADIUS, 2 * bench.RADIUS]}
    assert bench.fine_pass_kernel(FakeCtx([dict(fine, kernel="k_corr_tc")])) == "k_corr_tc"
    other = {"chip": [128, 128], "surface": [50, 50], "kernel": "k_corr_tc"}
    assert bench.fine_pass_kernel(FakeCtx([other])) == "k_corr_tc2"  # untuned: the fixed rule
    for k in ("k_corr_tc2", "k_corr_tc"):
        t = bench.profile_traffic(1000, k)
        assert t is not None and 500e3 < t < 2e6
    assert bench.profile_traffic(1000, "k_corr") is None
