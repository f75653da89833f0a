"""GPU preprocessing and quantisation (`_prepare`, src/api.jl:305-311) against the oracle.

For integer imagery every box sum is an exact FP64 integer, so the filtered Float32 image and
the eroded mask are bit-identical to the oracle's (the reference's banded running sums); the
UInt8 quantiser's global sums are reduced in double-double, so quantised pixels agree exactly
except for values within ~1e-13 of a rounding boundary (none expected; at most a handful
allowed, by one level). Float32 imagery of bounded dynamic range also sums exactly.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(ar, n=(600, 520), seed=3, holes=True):
    a, b, valid, _ = ar.synthetic.scale_u16_pair(640, seed=seed, max_amp=6.0)
    a = a[:n[0], :n[1]]
    b = b[:n[0], :n[1]]
    sv = valid[:n[0], :n[1]] if holes else None
    rv = np.ones(a.shape, bool)
    if holes:
        rv[100:130, 40:300] = False
    return a, b, rv, sv


def _check(ar, O, a, b, rv, sv, p, pre, width=5, min_std=0.0, quant="uint8", max_diff=0,
           rtol=0.0):
    got = ar.prepare(ar.ImagePair(a, b, rv, sv), p)
    gr, gs, grv, gsv = got.download()
    for img, mask, g, gm in ((a, rv, gr, grv), (b, sv, gs, gsv)):
        want, wm = O.prepare(img, mask, pre, width, min_std, quant)
        assert g.dtype == want.dtype
        assert np.array_equal(gm, wm)
        if g.dtype.kind == "f":
            same = (g == want) | (np.isnan(g) & np.isnan(want))
            if rtol:
                same |= np.abs(g - want) <= rtol * np.maximum(1.0, np.abs(want))
            assert np.count_nonzero(~same) <= max_diff, np.abs(g - want)[~same].max()
        else:
            d = np.abs(g.astype(np.int32) - want.astype(np.int32))
            assert d.max() <= (1 if max_diff else 0) and np.count_nonzero(d) <= max_diff


def test_highpass_uint8_default_pipeline(ar, O, gpu_lib):
    a, b, rv, sv = _pair(ar)
    _check(ar, O, a, b, rv, sv, ar.params(), "highpass", 5, quant="uint8", max_diff=2)


def test_highpass_no_quantize_exact(ar, O, gpu_lib):
    a, b, rv, sv = _pair(ar)
    _check(ar, O, a, b, rv, sv, ar.params(quantize="none"), "highpass", 5, quant="none")
    _check(ar, O, a, b, rv, sv, ar.params(quantize="none", filter_width=21), "highpass", 21,
           quant="none")


def test_wallis(ar, O, gpu_lib):
    a, b, rv, sv = _pair(ar, n=(300, 280))
    af, bf = a.astype(np.float32) / 65535, b.astype(np.float32) / 65535
    # Float32 local deviations span ~30 binades, so the FP64 box sums of d^2 can round
    # differently from the reference's running sums: agreement to 1e-5 relative.
    _check(ar, O, af, bf, rv, sv, ar.params(preprocess="wallis", quantize="none"), "wallis", 5,
           quant="none", rtol=1e-5)
    p = ar.params(preprocess=ar.Wallis(width=7, min_std=0.01), quantize="uint8")
    _check(ar, O, af, bf, rv, sv, p, "wallis", 7, 0.01, quant="uint8", max_diff=af.size // 1000)


def test_no_preprocess_paths(ar, O, gpu_lib):
    a, b, rv, sv = _pair(ar, n=(200, 190))
    _check(ar, O, a, b, rv, sv, ar.params(preprocess="none"), "none", quant="uint8", max_diff=2)
    f = a.astype(np.float32)
    f[5, 5] = np.nan
    f[7, 9] = np.inf
    g = ar.prepare(ar.ImagePair(f, f), ar.params(preprocess="none", quantize="none"))
    r, s, rm, sm = g.download()
    assert r[5, 5] == 0 and r[7, 9] == 0 and not rm[5, 5] and not rm[7, 9]
    assert np.array_equal(r[~np.isnan(f) & np.isfinite(f)], f[np.isfinite(f)])


def test_reference_known_answers(ar, gpu_lib):
    # test/preprocess.jl: a ramp is removed, a no-data band does not bias the local mean,
    # a uniform image quantises to mid-grey, an all-invalid image to zero.
    n = 40
    i, j = np.meshgrid(np.arange(1, n + 1), np.arange(1, n + 1), indexing="ij")
    ramp = (np.float32(0.01) * (i + 2 * j)).astype(np.float32)
    r, _, _, _ = ar.prepare(ar.ImagePair(ramp, ramp), ar.params(quantize="none")).download()
    assert np.abs(r[5:n - 5, 5:n - 5]).max() < 1e-4
    img = np.full((20, 20), 10.0, np.float32)
    m = np.ones((20, 20), bool)
    img[:5] = 0
    m[:5] = False
    r, _, rm, _ = ar.prepare(ar.ImagePair(img, img, m, m), ar.params(quantize="none")).download()
    assert abs(r[7, 9]) < 1e-4 and abs(r[6, 9]) < 1e-4 and not rm[2, 9]
    u = np.full((10, 10), 5.0, np.float32)
    q, _, _, _ = ar.prepare(ar.ImagePair(u, u), ar.params(preprocess="none")).download()
    assert np.all(q == 0x80)
    z = np.zeros((10, 10), bool)
    q, _, _, _ = ar.prepare(ar.ImagePair(u, u, z, z), ar.params(preprocess="none")).download()
    assert np.all(q == 0)


def test_filter_wider_than_image(ar, O, gpu_lib):
    a = np.random.default_rng(0).integers(0, 4000, (4, 30)).astype(np.uint16)
    _check(ar, O, a, a.copy(), None, None, ar.params(quantize="none", filter_width=7),
           "highpass", 7, quant="none")


def test_prepared_pair_tracks_like_host_prepared(ar, O, gpu_lib):
    """prepare on the device then track equals tracking the oracle-prepared images."""
    a, b, rv, sv = _pair(ar, n=(400, 400))
    p = ar.params()
    prep = ar.prepare(ar.ImagePair(a, b, rv, sv), p)
    pts = ar.gridpoints(a.shape, 16, chip_size=32, search_radius=12)
    got = ar.track(prep, pts, p)
    wr, wrm = O.prepare(a, rv, "highpass", 5)
    ws, wsm = O.prepare(b, sv, "highpass", 5)
    from conftest import fields
    want = O.track(wr, ws, fields(pts), upsampling=64, reference_valid=wrm, secondary_valid=wsm)
    g = (got.dx.ravel(order="F"), got.dy.ravel(order="F"), got.correlation.ravel(order="F"),
         got.searched.ravel(order="F"))
    for x, y in zip(g, want):
        same = (x == y) | (np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else (x == y)
        assert same.mean() > 0.995


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16, np.int16])
@pytest.mark.parametrize("width", [3, 5, 7, 9])
def test_highpass_small_widths_exact(ar, O, gpu_lib, dtype, width):
    """Square odd windows up to 9 on integer imagery (the warp-per-row-strip kernel): ragged
    extents (strip and column-block remainders), invalid blocks, single pixels and image edges
    against the oracle, bit for bit."""
    rng = np.random.default_rng(width)
    for shape in ((61, 70), (100, 129), (33, 5)):
        hi = {np.uint8: 256, np.uint16: 65536, np.int16: 32768}[dtype]
        lo = -32768 if dtype == np.int16 else 0
        a = rng.integers(lo, hi, shape).astype(dtype)
        m = rng.random(shape) > 0.05
        m[10:14, :] = False
        m[:, 3] = False
        p = ar.params(quantize="none", filter_width=width)
        _check(ar, O, a, a[::-1].copy(), m, m[::-1].copy(), p, "highpass", width, quant="none")
