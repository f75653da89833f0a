"""The request loop (ar_submit / ar_poll / ar_wait): continuous batching of autorift() requests.

Each request's result must be bit-identical to the same request run alone through the plain
path (ar_pair_upload, ar_prepare, ar_multichip one pair at a time), whatever it ran beside;
timeouts, polling, failures and a memory budget that admits one request at a time behave as
the header states.
"""

import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scenes(ar):
    out = []
    a, b, v, _ = ar.synthetic.scale_u16_pair(640, seed=3)
    out.append((a, b, v, dict(grid_spacing=16)))
    a, b, v, _ = ar.synthetic.scale_u16_pair(800, seed=4, max_amp=6.0)
    out.append((a, b, v, dict(grid_spacing=8, chip_size=16, search_radius=12, preprocess="wallis")))
    ref, sec = ar.synthetic.shifted_pair(512, (3.4, -2.2), seed=5, dtype=np.uint8)
    out.append((ref, sec, None, dict(grid_spacing=16, preprocess="none", quantize="none",
                                     chip_size=32, search_radius=20)))
    a, b, v, _ = ar.synthetic.scale_u16_pair(720, seed=6)
    out.append((a, b, v, dict(grid_spacing=12, chip_size=32, search_radius=(16), upsampling=16)))
    ref, sec = ar.synthetic.shifted_pair(448, (-1.3, 4.6), seed=7, dtype=np.float32)
    out.append((ref, sec, None, dict(grid_spacing=16, similarity="ncc")))
    return out


def same(x, y):
    for name in ("dx", "dy", "correlation"):
        a, b = getattr(x, name), getattr(y, name)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
    assert np.array_equal(x.chip_size, y.chip_size)
    assert np.array_equal(x.interpolated, y.interpolated)


@pytest.fixture(scope="module")
def cases(ar, gpu_lib):
    alone_ctx = ar._lib.Context(0)
    out = []
    for ref, sec, v, kw in scenes(ar):
        alone = ar.autorift(ref, sec, secondary_valid=v, ctx=alone_ctx, **kw)
        out.append((ref, sec, v, kw, alone))
    alone_ctx.close()
    return out


def test_results_identical_alone_and_in_the_mix(ar, cases):
    ctx = ar._lib.Context(0)
    ctx.set_option(ar._lib.AR_OPT_SERVE_SLOTS, 3)
    tickets = [None] * (2 * len(cases))

    def submit_from_thread(start):
        for k in range(start, len(tickets), 2):
            ref, sec, v, kw, _ = cases[k % len(cases)]
            tickets[k] = ar.submit(ref, sec, secondary_valid=v, ctx=ctx, **kw)

    threads = [threading.Thread(target=submit_from_thread, args=(s,)) for s in (0, 1)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for k, t in enumerate(tickets):
        same(t.wait(timeout=120), cases[k % len(cases)][4])
        q, r = t.times()
        assert q >= 0 and r > 0
        t.release()
    ctx.close()


def test_mixed_geometries_concurrently(ar, gpu_lib):
    """Many requests whose launches of the same kernels need different shared memory (chip
    16/32/64, radius 8..48) running at once in four slots: every result as alone."""
    a, b, v, _ = ar.synthetic.scale_u16_pair(512, seed=11)
    kinds = [dict(grid_spacing=16, chip_size=16, search_radius=8),
             dict(grid_spacing=16, chip_size=32, search_radius=25),
             dict(grid_spacing=16, chip_size=64, search_radius=10),
             dict(grid_spacing=32, chip_size=16, search_radius=48)]
    alone_ctx = ar._lib.Context(0)
    alone = [ar.autorift(a, b, secondary_valid=v, ctx=alone_ctx, **kw) for kw in kinds]
    alone_ctx.close()
    ctx = ar._lib.Context(0)
    ctx.set_option(ar._lib.AR_OPT_SERVE_SLOTS, 4)
    tickets = [ar.submit(a, b, secondary_valid=v, ctx=ctx, **kinds[k % len(kinds)])
               for k in range(24)]
    for k, t in enumerate(tickets):
        same(t.wait(timeout=120), alone[k % len(kinds)])
        t.release()
    ctx.close()


def test_timeout_poll_and_release(ar, gpu_lib):
    ctx = ar._lib.Context(0)
    a, b, v, _ = ar.synthetic.scale_u16_pair(1024, seed=8)
    t = ar.submit(a, b, secondary_valid=v, ctx=ctx, grid_spacing=8)
    with pytest.raises(TimeoutError):
        t.wait(timeout=0)  # just submitted: the upload alone takes longer
    while not t.done():
        pass
    r = t.wait(timeout=0)
    assert np.isfinite(r.dx).mean() > 0.5
    t.release()
    with pytest.raises(ar._lib.ArError):
        ctx.check(ctx.lib.ar_poll(ctx.handle, t.ticket, ar._lib.ctypes.byref(ar._lib.ctypes.c_int())))
    ctx.close()


def test_failed_request_reports_its_error(ar, gpu_lib):
    ctx = ar._lib.Context(0)
    ref, sec = ar.synthetic.shifted_pair(256, (1.0, 1.0), dtype=np.uint8)
    grid = ar.gridpoints(ref.shape, 16, chip_size=32, search_radius=8)
    bad = ar.points.PointSet(**{f: getattr(grid, f).copy() for f in ar.points.FIELDS})
    bad.x[0, 0] = np.nan  # rejected by the search: coordinates must be finite
    t = ar.submit(ref, sec, bad, ctx=ctx, preprocess="none", quantize="none")
    with pytest.raises(ar._lib.ArError, match="finite"):
        t.wait(timeout=60)
    ok = ar.submit(ref, sec, grid, ctx=ctx, preprocess="none", quantize="none")
    assert np.isfinite(ok.wait(timeout=60).dx).any()  # the loop carries on
    ctx.close()


def test_budget_of_one_request_runs_them_in_turn(ar, cases):
    ctx = ar._lib.Context(0)
    ctx.set_option(ar._lib.AR_OPT_SERVE_SLOTS, 4)
    ctx.set_option(ar._lib.AR_OPT_SERVE_MEMORY_MB, 1)  # below any request: one at a time
    tickets = [ar.submit(ref, sec, secondary_valid=v, ctx=ctx, **kw) for ref, sec, v, kw, _ in cases]
    for t, c in zip(tickets, cases):
        same(t.wait(timeout=120), c[4])
    with pytest.raises(ar._lib.ArError, match="already started"):
        ctx.set_option(ar._lib.AR_OPT_SERVE_SLOTS, 2)
    ctx.close()
