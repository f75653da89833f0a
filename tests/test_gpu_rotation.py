"""The rotation search on the GPU (ar_track_rotated, rotation in ar_multichip_params and
ar_request) against the oracle (src/track.jl:313-409).

Tolerances. A turned chip is a Float32 resample, so every element type correlates on the
FP32/FP64 path: correlation agrees with the oracle within 1e-5. Which angle wins depends on
peaks that may nearly tie, so the checks apply where the oracle's best and second-best angle
peaks differ by more than 1e-4 (the excluded share is small and bounded). There, integer
peaks agree and sub-pixel offsets agree within 1e-3 px except for near-ties of the 1/up
cascade argmax, whose rate is bounded as in the plain float parity tests.
"""

import ctypes

import numpy as np
import pytest

from conftest import fields
from test_oracle_multichip import mc_params

pytestmark = pytest.mark.gpu


def rotated_scene(ar, n=256, deg=2.5, seed=5, dtype=np.float32):
    a = ar.synthetic.synthetic_texture((n, n), seed=seed, dtype=np.float64)
    b = ar.synthetic.rotate_bilinear(a, deg)
    if np.dtype(dtype).kind == "f":
        return a.astype(dtype), b.astype(dtype)
    mx = np.iinfo(dtype).max
    q = lambda v: np.round(np.clip(v, 0, 1) * mx).astype(dtype)
    return q(a), q(b)


def angle_margin(O, ref, sec, pts, angs, measure="zncc", rv=None, sv=None):
    """Per point, the oracle's gap between the best and second-best angle peaks."""
    peaks = np.stack([O.track(ref, sec, fields(pts), upsampling=1, measure=measure,
                              reference_valid=rv, secondary_valid=sv, angles=(g,))[2]
                      for g in angs])
    peaks = np.where(np.isnan(peaks), -np.inf, peaks)
    if len(angs) == 1:
        return np.full(peaks.shape[1], np.inf)
    s = np.sort(peaks, axis=0)
    return s[-1] - s[-2]


def run_both(ar, O, ref, sec, pts, rot, up=16, measure="zncc", rv=None, sv=None):
    p = ar.params(preprocess="none", quantize="none", upsampling=up if up > 1 else 2,
                  similarity=measure, rotation=rot)
    sub = ar.NoRefine() if up == 1 else ar.PyramidRefine(up)
    got = ar.track(ar.ImagePair(ref, sec, rv, sv), pts, p, subpixel=sub)
    angs = ar.angles(p.rotation)
    want = O.track(ref, sec, fields(pts), upsampling=up, measure=measure, reference_valid=rv,
                   secondary_valid=sv, angles=angs)
    g = tuple(a.ravel(order="F") for a in (got.dx, got.dy, got.correlation, got.searched))
    return g, want, angle_margin(O, ref, sec, pts, angs, measure, rv, sv)


def check(g, w, margin, max_flip=0.02, max_close=0.05):
    gdx, gdy, gc, gs = g
    wdx, wdy, wc, ws = w
    assert np.array_equal(gs, ws)
    clear = margin > 1e-4
    close = ws & ~clear & np.isfinite(margin)
    assert close.sum() <= max(2, max_close * ws.sum()), f"{close.sum()} near-tied angles"
    m = clear & ~np.isnan(wdx)
    assert np.array_equal(np.isnan(gdx[clear]), np.isnan(wdx[clear]))
    assert m.sum() > 0
    assert np.abs(gc[m] - wc[m]).max() <= 1e-5
    d = np.maximum(np.abs(gdx[m] - wdx[m]), np.abs(gdy[m] - wdy[m]))
    flips = np.count_nonzero(d > 1e-3)
    assert flips <= max(1, max_flip * m.sum()), f"{flips} of {m.sum()} sub-pixel flips"
    return m.sum()


@pytest.mark.parametrize("dtype,up,measure", [
    (np.float32, 16, "zncc"), (np.float32, 1, "zncc"), (np.uint8, 64, "zncc"),
    (np.uint16, 16, "zncc"), (np.uint8, 16, "ncc"), (np.int16, 8, "zncc")])
def test_grid_parity(ar, O, gpu_lib, dtype, up, measure):
    ref, sec = rotated_scene(ar, dtype=dtype if dtype != np.int16 else np.uint16)
    if dtype == np.int16:
        ref, sec = (ref.astype(np.int32) - 32768).astype(np.int16), \
            (sec.astype(np.int32) - 32768).astype(np.int16)
    pts = ar.gridpoints(ref.shape, 14, chip_size=32, search_radius=8)
    g, w, mg = run_both(ar, O, ref, sec, pts, (-3.0, 0.0, 3.0), up=up, measure=measure)
    assert check(g, w, mg) > 100


def test_about_and_five_angles(ar, O, gpu_lib):
    ref, sec = rotated_scene(ar, deg=-4.0, seed=9, dtype=np.uint8)
    pts = ar.gridpoints(ref.shape, 16, chip_size=48, search_radius=6)
    rot = ar.RotationSearch((-4, -2, 0, 2, 4), about=-3.5)
    g, w, mg = run_both(ar, O, ref, sec, pts, rot, up=32)
    check(g, w, mg)


def test_scattered_points_padding_priors_masks(ar, O, gpu_lib):
    """Non-square chips (distinct row and column centres), zero padding at the border, priors
    and masks: the turned chip reads the padded secondary, zero outside the image."""
    rng = np.random.default_rng(3)
    ref, sec = rotated_scene(ar, n=200, deg=3.0, seed=11, dtype=np.float32)
    n = 300
    pts = ar.pointset(rng.uniform(-5, 206, n), rng.uniform(-5, 206, n),
                      chip_size=rng.choice([16, 20, 32], n), chip_size_y=rng.choice([16, 24, 32], n),
                      search_radius_x=rng.integers(0, 10, n), search_radius_y=rng.integers(1, 10, n),
                      dx_prior=np.round(rng.normal(0, 3, n)), dy_prior=rng.normal(0, 2, n))
    rv = np.ones(ref.shape, bool)
    rv[60:90, 20:70] = False
    sv = np.ones(ref.shape, bool)
    sv[:, 160:] = False
    g, w, mg = run_both(ar, O, ref, sec, pts, (-2.0, 0.0, 2.5), up=16, rv=rv, sv=sv)
    assert w[3].any() and (~w[3]).any()
    check(g, w, mg, max_close=0.08)


def test_large_chip(ar, O, gpu_lib):
    ref, sec = rotated_scene(ar, n=400, deg=3.0, seed=2, dtype=np.uint8)
    pts = ar.gridpoints(ref.shape, 60, chip_size=128, search_radius=25)
    g, w, mg = run_both(ar, O, ref, sec, pts, (-3.0, 3.0), up=16)
    check(g, w, mg, max_close=0.2)


def test_degenerate_angles(ar, O, gpu_lib):
    zero = np.zeros((120, 120), np.uint8)
    flat = np.full((120, 120), 7, np.uint8)
    pts = ar.gridpoints(zero.shape, 30, chip_size=16, search_radius=5)
    for img in (zero, flat):
        g, w, _ = run_both(ar, O, img, img, pts, (-3.0, 0.0, 3.0), up=16)
        assert np.array_equal(g[3], w[3]) and g[3].all()
        assert np.array_equal(np.isnan(g[0]), np.isnan(w[0]))
    assert np.isnan(g[0]).sum() == 0  # a turned flat chip has zero corners: measured
    p = ar.params(preprocess="none", quantize="none", rotation=(0.0,))
    d = ar.track(ar.ImagePair(flat, flat), pts, p)
    assert d.searched.all() and np.isnan(d.dx).all()


@pytest.mark.parametrize("dtype", [np.float32, np.uint16])
def test_single_zero_angle_bit_identical_to_plain(ar, gpu_lib, dtype):
    """test/firstguess.jl:289-307: RotationSearch((0.0,)) correlates the chip itself; for these
    element types the two passes run the same arithmetic, so every output is identical."""
    ref, sec = ar.synthetic.shifted_pair(256, (4, -3), seed=2, dtype=dtype)
    pts = ar.gridpoints(ref.shape, 16, chip_size=32, search_radius=10)
    pair = ar.ImagePair(ref, sec)
    off = ar.track(pair, pts, ar.params(preprocess="none", quantize="none"))
    one = ar.track(pair, pts, ar.params(preprocess="none", quantize="none", rotation=(0.0,)))
    for name in ("dx", "dy", "correlation"):
        a, b = getattr(off, name), getattr(one, name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
    assert np.array_equal(off.searched, one.searched)


def test_single_zero_angle_uint8_displacements(ar, gpu_lib):
    """UInt8: the plain pass's numerator is exact, the search's FP32/FP64; displacements agree."""
    ref, sec = ar.synthetic.shifted_pair(256, (4, -3), seed=2, dtype=np.uint8)
    pts = ar.gridpoints(ref.shape, 16, chip_size=32, search_radius=10)
    pair = ar.ImagePair(ref, sec)
    off = ar.track(pair, pts, ar.params(preprocess="none", quantize="none"))
    one = ar.track(pair, pts, ar.params(preprocess="none", quantize="none", rotation=(0.0,)))
    m = ~np.isnan(off.dx)
    assert np.array_equal(m, ~np.isnan(one.dx))
    d = np.maximum(np.abs(off.dx - one.dx), np.abs(off.dy - one.dy))[m]
    assert np.count_nonzero(d > 1e-3) <= max(1, 0.02 * m.sum())
    assert np.abs(off.correlation[m] - one.correlation[m]).max() <= 1e-6


def test_multichip_default_pipeline(ar, O, gpu_lib):
    """autorift's search with rotation = true (every level, coarse passes included) against the
    oracle on the same prepared pair."""
    a, b = rotated_scene(ar, n=384, deg=2.0, seed=4, dtype=np.uint16)
    p = ar.params(grid_spacing=16, rotation=True)
    prep = ar.prepare(ar.ImagePair(a, b), p)
    grid = ar.build_grid(a.shape, p)
    got = ar.correlate_multichip(prep, grid, p)
    wr, wrm = O.prepare(a, None, "highpass", 5)
    ws, wsm = O.prepare(b, None, "highpass", 5)
    want = O.multichip(wr, ws, fields(grid), mc_params(ar, p), wrm, wsm,
                       angles=ar.angles(p.rotation))
    gdx, wdx = got.dx, want[0]
    both = ~np.isnan(gdx) & ~np.isnan(wdx)
    assert both.mean() > 0.7
    assert np.count_nonzero(np.isnan(gdx) != np.isnan(wdx)) <= 0.03 * gdx.size
    d = np.maximum(np.abs(gdx - wdx), np.abs(got.dy - want[1]))[both]
    assert np.count_nonzero(d > 1e-3) <= 0.03 * both.sum()
    assert np.count_nonzero(got.chip_size != want[3]) <= 0.03 * gdx.size


def test_rotation_search_recovers_correlation(ar, gpu_lib):
    """test/firstguess.jl:309-330 on the GPU: median correlation at least 5% higher."""
    n = 256
    a = ar.synthetic.synthetic_texture((n, n), seed=5)
    b = ar.synthetic.rotate_bilinear(a, 3.0)
    kw = dict(chip_size=32, chip_size_max=32, search_radius=8, quantize="none", outliers="none")
    plain = ar.autorift(a, b, **kw)
    rot = ar.autorift(a, b, rotation=ar.RotationSearch((-3.0, 0.0, 3.0)), **kw)
    cp = np.median(plain.correlation[~np.isnan(plain.correlation)])
    cr = np.median(rot.correlation[~np.isnan(rot.correlation)])
    assert cr > 1.05 * cp, (cp, cr)


def test_serving_identical_to_alone(ar, gpu_lib):
    a, b = rotated_scene(ar, n=320, deg=2.0, seed=6, dtype=np.uint16)
    kw = dict(grid_spacing=16, rotation=(-2.0, 0.0, 2.0))
    alone = ar.autorift(a, b, **kw)
    ctx = ar._lib.Context(0)
    ctx.set_option(ar._lib.AR_OPT_SERVE_SLOTS, 2)
    ts = [ar.submit(a, b, ctx=ctx, **kw), ar.submit(a, b, ctx=ctx, grid_spacing=16),
          ar.submit(a, b, ctx=ctx, **kw)]
    for k in (0, 2):
        r = ts[k].wait(timeout=120)
        for name in ("dx", "dy", "correlation"):
            assert np.array_equal(getattr(r, name).view(np.uint32),
                                  getattr(alone, name).view(np.uint32)), name
    ts[1].wait(timeout=120)
    for t in ts:
        t.release()
    ctx.close()


def test_invalid_angles_are_rejected(ar, gpu_lib):
    ctx = ar._lib.default_context()
    ref, sec = ar.synthetic.shifted_pair(64, (1, 1), dtype=np.uint8)
    pair = ar.ImagePair(ref, sec).device(ctx)
    pts = ar.gridpoints(ref.shape, 16, chip_size=16, search_radius=4)
    from autorift_b200.track import points_struct
    st, keep = points_struct(pts)
    n = len(pts)
    outs = [np.empty(n, np.float32) for _ in range(3)] + [np.empty(n, np.uint8)]
    for angs in ([0.0, float("nan")], [1.0, 1.0], list(range(65)), [float("inf")]):
        a = np.asarray(angs, np.float64)
        rc = ctx.lib.ar_track_rotated(ctx.handle, pair.handle, ctypes.byref(st), 16, 0,
                                      a.ctypes.data, a.size, *(o.ctypes.data for o in outs))
        assert rc == 1, angs  # AR_ERR_ARG
    rc = ctx.lib.ar_track_rotated(ctx.handle, pair.handle, ctypes.byref(st), 16, 0,
                                  None, 3, *(o.ctypes.data for o in outs))
    assert rc == 1
    prm = ar.multichip_params(ar.params())
    bad = np.array([0.0, np.nan])
    prm.rotation_count, prm.rotation_angles = 2, bad.ctypes.data
    gs, gr, gc = st, *pts.shape
    o5 = [np.empty(gr * gc, np.float32) for _ in range(3)] + [np.empty(gr * gc, np.uint16),
                                                             np.empty(gr * gc, np.uint8)]
    rc = ctx.lib.ar_multichip(ctx.handle, pair.handle, ctypes.byref(gs), gr, gc,
                              ctypes.byref(prm), *(o.ctypes.data for o in o5))
    assert rc == 1


def test_device_entry_matches_host_entry(ar, gpu_lib):
    """ar_track_device_rotated (device points and outputs) gives ar_track_rotated's results."""
    import torch
    ctx = ar._lib.default_context()
    ref, sec = rotated_scene(ar, n=256, deg=2.0, seed=12, dtype=np.uint8)
    pts = ar.gridpoints(ref.shape, 12, chip_size=32, search_radius=8)
    p = ar.params(preprocess="none", quantize="none", rotation=True)
    pair = ar.ImagePair(ref, sec)
    host = ar.track(pair, pts, p, ctx=ctx)
    from autorift_b200.points import FIELDS
    dev = torch.device("cuda", 0)
    cols = {f: torch.from_numpy(pts.flat(f)).to(dev) for f in FIELDS}
    st = ar._lib.ArPoints(*(cols[f].data_ptr() for f in FIELDS), len(pts))
    n = len(pts)
    outs = [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3)]
    srch = torch.empty(n, dtype=torch.uint8, device=dev)
    angs = np.asarray(ar.angles(p.rotation), np.float64)
    ctx.check(ctx.lib.ar_track_device_rotated(
        ctx.handle, pair.device(ctx).handle, ctypes.byref(st), 64, 0, angs.ctypes.data,
        angs.size, *(o.data_ptr() for o in outs), srch.data_ptr(), None))
    ctx.check(ctx.lib.ar_synchronize(ctx.handle))
    for got, want in zip(outs, (host.dx, host.dy, host.correlation)):
        assert np.array_equal(got.cpu().numpy().view(np.uint32),
                              want.ravel(order="F").view(np.uint32))
    assert np.array_equal(srch.cpu().numpy().astype(bool), host.searched.ravel(order="F"))
