"""GPU parity: the sm_100a library through its C ABI against the CPU oracle.

Tolerances.
  * UInt8 imagery (the default pipeline's element type) with a power-of-two chip area (every
    chip-size level of the default search) is exact: the mean-removed chip is then exactly
    representable in Float32, the numerator is an exact integer sum, the denominator exact
    integer box sums with the same rounded FP64 operations, the cascade the same Float32
    operations. dx, dy, correlation and searched must be bit-identical to the oracle.
  * UInt8 with any other chip area: the oracle rounds the mean-removed chip to Float32 before
    its FP64 sum while the GPU sums the exact integers, so correlation agrees within 1e-6 and
    sub-pixel offsets agree except near-ties.
  * UInt16 and Float32 numerators are FP32 products accumulated in FP32 over two chip columns
    and then in FP64 (the plain method). Correlation agrees within 1e-5; integer peaks agree
    wherever the oracle's top-two margin exceeds 1e-4; sub-pixel offsets agree within 1e-3 px
    except where the surfaces' last-bit differences flip a near-tie of the 1/up-quantised
    cascade argmax, whose rate is bounded and reported.
"""

import numpy as np
import pytest

from conftest import fields

pytestmark = pytest.mark.gpu


def run_both(ar, O, ref, sec, pts, up=64, measure="zncc", rv=None, sv=None):
    p = ar.params(preprocess="none", quantize="none", upsampling=up if up > 1 else 2,
                  similarity=measure)
    sub = ar.NoRefine() if up == 1 else ar.PyramidRefine(up)
    got = ar.track(ar.ImagePair(ref, sec, rv, sv), pts, p, subpixel=sub)
    want = O.track(ref, sec, fields(pts), upsampling=up, measure=measure, reference_valid=rv,
                   secondary_valid=sv)
    g = tuple(a.ravel(order="F") for a in (got.dx, got.dy, got.correlation, got.searched))
    return g, want


def assert_identical(g, w):
    for a, b, name in zip(g, w, ("dx", "dy", "correlation", "searched")):
        assert a.shape == b.shape
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        assert same.all(), f"{name}: {np.count_nonzero(~same)} of {a.size} differ"


def assert_close_u8(g, w, max_flip=0.03):
    """Non-power-of-two chip areas: correlation within 1e-6, near-tie flips bounded."""
    gdx, gdy, gc, gs = g
    wdx, wdy, wc, ws = w
    assert np.array_equal(gs, ws)
    m = ~np.isnan(wdx)
    assert np.array_equal(m, ~np.isnan(gdx))
    assert np.abs(gc[m] - wc[m]).max() <= 1e-6
    d = np.maximum(np.abs(gdx[m] - wdx[m]), np.abs(gdy[m] - wdy[m]))
    assert np.count_nonzero(d > 0) <= max(1, max_flip * m.sum())


@pytest.mark.parametrize("chip,radius,spacing,up", [
    (32, 25, 16, 64), (32, 10, 12, 16), (16, 6, 9, 8), (64, 25, 24, 64), (32, 25, 16, 1),
    (32, 3, 10, 2), (128, 12, 40, 32)])
def test_uint8_grid_bit_identical(ar, O, gpu_lib, chip, radius, spacing, up):
    ref, sec = ar.synthetic.shifted_pair(320, (4.4, -2.7), seed=chip + radius, dtype=np.uint8)
    pts = ar.gridpoints(ref.shape, spacing, chip_size=chip, search_radius=radius)
    g, w = run_both(ar, O, ref, sec, pts, up=up)
    assert w[3].any()
    assert_identical(g, w)


@pytest.mark.parametrize("chip,radius,spacing,up", [(24, 7, 10, 4), (20, 9, 11, 16), (48, 14, 20, 64)])
def test_uint8_grid_non_power_of_two_chip(ar, O, gpu_lib, chip, radius, spacing, up):
    ref, sec = ar.synthetic.shifted_pair(320, (4.4, -2.7), seed=chip + radius, dtype=np.uint8)
    pts = ar.gridpoints(ref.shape, spacing, chip_size=chip, search_radius=radius)
    g, w = run_both(ar, O, ref, sec, pts, up=up)
    assert w[3].any()
    assert_close_u8(g, w)


def test_uint8_scattered_padding_priors_masks(ar, O, gpu_lib):
    rng = np.random.default_rng(3)
    ref, sec = ar.synthetic.shifted_pair(256, (6.25, 3.5), seed=9, dtype=np.uint8)
    n = 400
    x = rng.uniform(-5, 262, n)
    y = rng.uniform(-5, 262, n)
    pts = ar.pointset(x, y, chip_size=rng.choice([16, 20, 32, 48], n),
                      chip_size_y=rng.choice([16, 24, 32], n),
                      search_radius_x=rng.integers(0, 20, n), search_radius_y=rng.integers(1, 20, n),
                      dx_prior=np.round(rng.normal(0, 4, n)), dy_prior=rng.normal(0, 3, n))
    rv = np.ones(ref.shape, bool)
    rv[100:140, 30:90] = False
    sv = np.ones(ref.shape, bool)
    sv[:, 200:] = False
    g, w = run_both(ar, O, ref, sec, pts, up=16, rv=rv, sv=sv)
    assert w[3].any() and (~w[3]).any()
    assert_close_u8(g, w)
    # Points whose chip area is a power of two are exact.
    area = (2 * (pts.chip_size_x // 2)) * (2 * (pts.chip_size_y // 2))
    p2 = (area & (area - 1)) == 0
    assert p2.sum() > 50
    assert_identical(tuple(a[p2] for a in g), tuple(a[p2] for a in w))


def test_uint8_degenerate_and_unsearched(ar, O, gpu_lib):
    ref, sec = ar.synthetic.shifted_pair(300, (0, 0), dtype=np.uint8)
    ref = ref.copy(); sec = sec.copy()
    ref[99:200, 99:200] = 128
    sec[99:200, 99:200] = 128
    pts = ar.gridpoints((300, 300), 32, chip_size=32, search_radius=25)
    pts.radius_x[1, 1] = 0
    g, w = run_both(ar, O, ref, sec, pts)
    assert_identical(g, w)
    S = g[3].reshape(pts.shape, order="F")
    DX = g[0].reshape(pts.shape, order="F")
    assert not S[1, 1] and np.isnan(DX[1, 1])
    flat = (pts.x >= 130) & (pts.x <= 170) & (pts.y >= 130) & (pts.y <= 170)
    assert S[flat].all() and np.isnan(DX[flat]).all()


def test_uint8_ncc(ar, O, gpu_lib):
    ref, sec = ar.synthetic.shifted_pair(200, (2, 1), seed=4, dtype=np.uint8)
    pts = ar.gridpoints(ref.shape, 16, chip_size=32, search_radius=10)
    g, w = run_both(ar, O, ref, sec, pts, up=16, measure="ncc")
    assert_identical(g, w)


def _float_checks(g, w, max_flip=0.02):
    gdx, gdy, gc, gs = g
    wdx, wdy, wc, ws = w
    assert np.array_equal(gs, ws)
    m = ~np.isnan(wdx)
    assert np.array_equal(m, ~np.isnan(gdx))
    assert np.abs(gc[m] - wc[m]).max() <= 1e-5
    d = np.maximum(np.abs(gdx[m] - wdx[m]), np.abs(gdy[m] - wdy[m]))
    flips = np.count_nonzero(d > 1e-3)
    assert flips <= max(1, max_flip * m.sum()), f"{flips} of {m.sum()} sub-pixel flips"
    assert d.max() <= 3 / 64 + 1e-9
    return flips / max(1, m.sum())


def test_float32_plain_512(ar, O, gpu_lib):
    a, b, (dx, dy) = ar.synthetic.plain_512_pair()
    pts = ar.synthetic.plain_512_points()
    g, w = run_both(ar, O, a, b, pts, up=64)
    rate = _float_checks(g, w)
    inner = np.isfinite(g[0])
    assert abs(np.median(-g[0][inner]) - dx) < 0.05
    assert abs(np.median(-g[1][inner]) - dy) < 0.05
    print(f"float32 sub-pixel flip rate {rate:.4f}")


def test_uint16_grid(ar, O, gpu_lib):
    ref, sec = ar.synthetic.shifted_pair(300, (3.3, -5.6), seed=21, dtype=np.uint16)
    pts = ar.gridpoints(ref.shape, 12, chip_size=32, search_radius=12)
    g, w = run_both(ar, O, ref, sec, pts, up=64)
    _float_checks(g, w)


@pytest.mark.parametrize("dtype", [np.float32, np.uint16])
def test_float_scattered_padding_priors_masks(ar, O, gpu_lib, dtype):
    """Points beyond the image edge: windows partly or wholly in the zero padding. A window
    without variance must give a zero surface value, as the oracle's exact sums do, never an
    arbitrary one."""
    rng = np.random.default_rng(3)
    ref, sec = ar.synthetic.shifted_pair(200, (2.5, -1.5), seed=11, dtype=dtype)
    n = 300
    pts = ar.pointset(rng.uniform(-5, 206, n), rng.uniform(-5, 206, n),
                      chip_size=rng.choice([16, 20, 32], n), chip_size_y=rng.choice([16, 24, 32], n),
                      search_radius_x=rng.integers(0, 10, n), search_radius_y=rng.integers(1, 10, n),
                      dx_prior=np.round(rng.normal(0, 3, n)), dy_prior=rng.normal(0, 2, n))
    rv = np.ones(ref.shape, bool)
    rv[60:90, 20:70] = False
    sv = np.ones(ref.shape, bool)
    sv[:, 160:] = False
    for up in (1, 16):
        g, w = run_both(ar, O, ref, sec, pts, up=up, rv=rv, sv=sv)
        assert np.nanmax(np.abs(g[2])) <= 1.0 + 1e-6
        _float_checks(g, w)


def test_integer_peaks_match_where_margin_is_clear(ar, O, gpu_lib):
    """Float32 surfaces: identical integer peaks wherever the oracle's top-two margin > 1e-4."""
    a, b, _ = ar.synthetic.plain_512_pair(seed=5)
    rng = np.random.default_rng(0)
    checked = 0
    for _ in range(40):
        cy, cx = rng.integers(60, 450, 2)
        chip = b[cy - 16:cy + 16, cx - 16:cx + 16]
        win = a[cy - 16 - 20:cy + 16 + 19, cx - 16 - 20:cx + 16 + 19]
        so, _ = O.correlate(win, chip, 20)
        sg, _ = ar.correlate(win, chip, 20)
        assert np.abs(sg - so).max() <= 1e-5
        top = np.sort(so.ravel())[-2:]
        if top[1] - top[0] > 1e-4:
            assert O.peak_index(sg) == O.peak_index(so)
            checked += 1
    assert checked > 20


def test_surfaces_vs_reference_fixtures(ar, O, gpu_lib, ref_golden):
    worst = 0.0
    for case in ref_golden.cases("matchtemplate__zncc"):
        a = ref_golden[case]
        r = ref_golden.meta[case]["search_radius"]
        sg, deg = ar.correlate(a["search"], a["chip"], r)
        so, _ = O.correlate(a["search"], a["chip"], r)
        assert not deg
        if "lowcontrast" in case:
            assert O.peak_index(sg) == (r, r)
            assert abs(float(sg.max()) - 1) <= 1e-3
            continue
        worst = max(worst, float(np.abs(sg - a["expected"]).max()))
        assert O.peak_index(sg) == O.peak_index(a["expected"]), case
        if a["chip"].dtype == np.uint8:
            assert np.array_equal(sg, so), case
        else:
            assert np.abs(sg - so).max() <= 1e-5, case
    assert worst < 1e-4


def test_surfaces_vs_opencv_golden(ar, O, gpu_lib, cv_golden):
    for case in cv_golden.meta["cases"]:
        a = cv_golden[case["name"]]
        sg, _ = ar.correlate(a["search"], a["chip"], (case["rx"], case["ry"]))
        assert np.abs(sg - a["expected"]).max() < 1e-4
        assert O.peak_index(sg) == tuple(case["shift_rc"])


def test_degenerate_surface_flag(ar, gpu_lib):
    win = np.random.default_rng(0).integers(0, 255, (51, 51)).astype(np.uint8)
    s, deg = ar.correlate(win, np.full((32, 32), 7, np.uint8), 10)
    assert deg and np.all(s == 0)


@pytest.mark.parametrize("up", [2, 4, 8, 16, 32, 64, 128])
def test_cascade_bit_identical(ar, O, gpu_lib, up):
    rng = np.random.default_rng(up)
    patches = rng.standard_normal((64, 5, 5)).astype(np.float32)
    patches[0] = 0.5
    patches[1] = 0
    patches[1, 2, 2] = 1
    patches[2] = np.round(patches[2])  # plateaus and ties
    row, col, val = ar.refine_patches(patches, up)
    for k in range(len(patches)):
        cur = patches[k]
        for _ in range(int(np.log2(up))):
            cur = O.pyrup(cur)
        i, j = O.peak_index(cur)
        assert (row[k], col[k]) == (i, j), k
        assert val[k] == cur[i, j]


def test_empty_and_unsearchable_sets(ar, gpu_lib):
    ref, sec = ar.synthetic.shifted_pair(100, (1, 1), dtype=np.uint8)
    pair = ar.ImagePair(ref, sec)
    pts = ar.pointset(np.zeros(0), np.zeros(0))
    d = ar.track(pair, pts)
    assert len(d) == 0
    pts = ar.pointset([50.0, 60.0], [50.0, 60.0], search_radius=0)
    d = ar.track(pair, pts)
    assert not d.searched.any() and np.isnan(d.dx).all()


def test_pair_ready_orders_other_streams(ar, gpu_lib):
    """ar_pair_upload and ar_prepare return once queued; a track on another stream right after
    them must still see the complete pair (the pair's ready event orders it)."""
    import ctypes

    import torch
    L = ar._lib
    ctx = L.Context(0)
    lib = ctx.lib
    a, b = ar.synthetic.shifted_pair(1024, (3.2, -1.7), seed=8, dtype=np.uint16)
    pts = ar.gridpoints(a.shape, 16, chip_size=32, search_radius=12)
    p = ar.params()
    want = ar.track(ar.prepare(ar.ImagePair(a, b), p, ctx), pts, p, ctx=ctx)
    from autorift_b200.points import FIELDS
    dev = torch.device("cuda", 0)
    side = torch.cuda.Stream(device=dev)
    cols = {f: torch.from_numpy(pts.flat(f)).to(dev) for f in FIELDS}
    torch.cuda.synchronize()
    st = L.ArPoints(*(cols[f].data_ptr() for f in FIELDS), len(pts))
    n = len(pts)
    outs = [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3)]
    srch = torch.empty(n, dtype=torch.uint8, device=dev)
    fa, fb = np.asfortranarray(a), np.asfortranarray(b)
    for _ in range(3):
        raw, prep = ctypes.c_void_p(), ctypes.c_void_p()
        ctx.check(lib.ar_pair_upload(ctx.handle, fa.ctypes.data, fb.ctypes.data, None, None,
                                     a.shape[0], a.shape[1], L.AR_U16, ctypes.byref(raw)))
        ctx.check(lib.ar_prepare(ctx.handle, raw, ctypes.byref(ar.prepare_options(p)),
                                 ctypes.byref(prep)))
        lib.ar_pair_destroy(raw)
        ctx.check(lib.ar_track_device(ctx.handle, prep, ctypes.byref(st), 64, L.AR_ZNCC,
                                      *(o.data_ptr() for o in outs), srch.data_ptr(),
                                      ctypes.c_void_p(side.cuda_stream)))
        side.synchronize()
        lib.ar_pair_destroy(prep)
        for got, w in zip(outs, (want.dx, want.dy, want.correlation)):
            assert np.array_equal(got.cpu().numpy().view(np.uint32),
                                  w.ravel(order="F").view(np.uint32))
    ctx.close()
