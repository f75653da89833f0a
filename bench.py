#!/usr/bin/env python
"""Benchmark: points/s of AutoRIFT.jl's default pipeline at chip 32 / radius 25 on B200.

Workload (one step): `autorift(image1, image2; grid_spacing=8)` with the reference's defaults
(src/api.jl:210-274) on a 10980^2 synthetic UInt16 pair (a Sentinel-2 tile's size): highpass
(width 5) and UInt8 quantisation of both images (src/api.jl:305-311), then the multi-chip-size
search (src/multichip.jl:106-422) over the 1350 x 1350 grid (spacing 8, margin from
chip_size_max 128) at chip sizes 32/64/128, search radius 25, PyramidRefine(64), ZNCC, Gardner
outlier filter and hole filling. Scene: seeded filtered noise (sigma 2, mean 8000, std 1500)
and its bicubic warp by a 6-bump field up to 15 px, 2% noise, 3% no-data blobs passed as the
secondary's mask.

`value` times the device work with the raw pair and the grid resident in HBM; `e2e` times the
same pipeline through the C ABI from host buffers (pair upload, grid upload, result download):
its value through the request loop (ar_submit, pairs overlapping on the device), its p50/p99
pair latency and `one_pair_at_a_time` through ar_pair_upload / ar_prepare / ar_multichip.
`plain_gpu_path` is the same step with the direct FP32 correlation on CUDA cores, one pair at a
time; `batched_vs_plain` sets the served rate against it. L2 (126 MB) is flushed before every
timed step by writing a 256 MiB buffer. The 4096^2 pair of the at-scale configuration (490 x
490 grid) is timed the same way and reported under `config_4096`; the serving configuration's
Poisson sweep (sides 512/2048/4096/10980 in 8:4:2:1) under `serving`.

Arms:
  default            our library (libautorift_gpu.so, sm_100a); N GPUs run N independent
                     replicas (one pair per rank, no collective on the data path).
  --impl reference   the reference's algorithm on the host cores: Julia is not installed, so
                     the CPU restatement (oracle/, C++ + OpenMP, all host threads) runs the
                     same pipeline on a centred 2048^2 crop of the scene per step.

Prints one JSON line (rank 0).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "points/sec at chip32/r25 vs plain GPU path; p50/p99 pair latency"
UNIT = "points/s"
N, SPACING, CHIP, RADIUS, UP = 10980, 8, 32, 25, 64
N_SCALE = 4096  # the at-scale configuration's pair, reported beside the headline
CROP = 2048  # host sample: the same pipeline on a centred crop of the scene
SERVE_RATES = (5, 10, 20, 50, 100, 200)  # pairs/s of the serving sweep


def workload(n, gr, gc):
    return (f"autorift() default pipeline (highpass 5, UInt8, multichip 32/64/128, Gardner, "
            f"fill) on a {n}^2 synthetic UInt16 pair, {gr}x{gc} grid spacing {SPACING}, radius "
            f"{RADIUS}, PyramidRefine({UP})")


def scene(ar, n=N, field=False):
    """The benchmark pair of side n; with `field`, also the imposed motion downsampled 4x."""
    a, b, valid, (fx, fy) = ar.synthetic.scale_u16_pair(n)
    if field:
        return a, b, valid, (np.ascontiguousarray(fx[::4, ::4]), np.ascontiguousarray(fy[::4, ::4]))
    return a, b, valid


def pipeline_params(ar, spacing=SPACING):
    return ar.params(grid_spacing=spacing, chip_size=CHIP, search_radius=RADIUS, upsampling=UP)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def replicas_rate(dist, elapsed_ms, points_per_rank, steps, device=None):
    """Whole-job rate of independent replicas: every rank processed `points_per_rank` points per
    step for `steps` steps; the job took as long as its slowest rank (max over ranks; no data
    moves between ranks). Returns (max elapsed ms, points/s of the whole job)."""
    import torch
    world = dist.get_world_size() if dist else 1
    t = torch.tensor([float(elapsed_ms)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    return ms, world * points_per_rank * steps / (ms * 1e-3)


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        return {}


def measure_fp32_peak(torch, device):
    """cuBLAS SGEMM with TF32 disabled: the measured FP32 CUDA-core rate (TFLOP/s)."""
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device=device, dtype=torch.float32)
    b = torch.randn(n, n, device=device, dtype=torch.float32)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


def profile_traffic(points, kernel):
    """DRAM bytes of one correlation launch of `kernel` over `points` searched points, from the
    committed ncu capture of the same kernel on the same pass geometry (bytes per point measured
    on a smaller grid); None when there is no capture of it."""
    f = ROOT / "profiles" / "k_corr_traffic.json"
    try:
        d = json.loads(f.read_text())
        return float(d[kernel]["bytes_per_point"]) * points
    except (OSError, ValueError, TypeError, KeyError):
        return None


def fine_pass_kernel(ctx):
    """The kernel the autotuner kept for the fine chip-32 / radius-25 pass (surface 50 x 50)."""
    for t in ctx.tuned():
        if t["chip"] == [CHIP, CHIP] and t["surface"] == [2 * RADIUS, 2 * RADIUS]:
            return t["kernel"]
    return "k_corr_tc2"


def crop(a, n):
    r0 = (a.shape[0] - n) // 2
    return np.ascontiguousarray(a[r0:r0 + n, r0:r0 + n])


def oracle_params(ar, p):
    """The oracle's multichip parameter dict for a Params."""
    o = p.outliers
    g = isinstance(o, ar.GardnerFilter)
    return dict(chip_base=p.chip_size_base, chip_min=p.chip_size_min, chip_max=p.chip_size_max,
                aspect=p.chip_aspect, min_radius=p.min_search_radius, stride=p.coarse_stride,
                buffer=p.coarse_buffer, min_frac=p.min_coarse_valid_fraction,
                up=ar.upsampling(p.subpixel), measure=0, outliers=1 if g else 0,
                window=o.window if g else 5, iterations=o.iterations if g else 3,
                min_agree_fraction=o.min_agree_fraction if g else 0.32,
                agree_tolerance=o.agree_tolerance if g else 0.2,
                mad_scale=o.mad_scale if g else 4.0, fill_window=p.fill_window)


def host_pipeline(O, ar, a, b, valid, p):
    """The oracle's pipeline on the host cores (prepare both images, multichip over the
    default grid); returns (grid points, seconds, multichip outputs, prepared images)."""
    grid = ar.build_grid(a.shape, p)
    fields = {f: getattr(grid, f) for f in ar.points.FIELDS}
    t = time.perf_counter()
    wr, wrm = O.prepare(a, None, "highpass", p.preprocess.width)
    ws, wsm = O.prepare(b, valid, "highpass", p.preprocess.width)
    out = O.multichip(wr, ws, fields, oracle_params(ar, p), wrm, wsm)
    return len(grid), time.perf_counter() - t, out, (wr, ws, wrm, wsm)


def crop_parity(ar, ctx, O, a, b, valid, p):
    """The whole pipeline on a centred CROP^2 crop of the scene, on the host cores (the oracle,
    timed: the CPU baseline) and through the library (`autorift` on the same crop, same grid
    rule): every output of every grid point compared bit for bit."""
    ca, cb, cv = crop(a, CROP), crop(b, CROP), crop(valid, CROP)
    pts, dt, want, prepared = host_pipeline(O, ar, ca, cb, cv, p)
    got = ar.autorift(ca, cb, secondary_valid=cv, ctx=ctx, grid_spacing=SPACING, chip_size=CHIP,
                      search_radius=RADIUS, upsampling=UP)
    names = ("dx", "dy", "correlation", "chip_size", "interpolated")
    gv = (got.dx, got.dy, got.correlation, got.chip_size, got.interpolated)
    same = {}
    for nm, g, w in zip(names, gv, want):
        g, w = np.asarray(g), np.asarray(w)
        if g.dtype.kind == "f":
            same[nm] = bool(np.array_equal(g.view(np.uint32), w.astype(np.float32).view(np.uint32)))
        else:
            same[nm] = bool(np.array_equal(g.astype(np.int64), w.astype(np.int64)))
    cpu = {"value": pts / dt, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
           "sample": f"the same pipeline on a centred {CROP}^2 crop ({pts} grid points), "
                     f"{dt:.1f} s",
           "numerator": "FP64 direct sum (the reference computes it with single-precision "
                        "FFTW, not installed here; the oracle is the exact value that "
                        "approximates)"}
    parity = {"crop": [CROP, CROP], "points": pts,
              "what": "the library's autorift() on the crop against the oracle's prepare + "
                      "multichip, every grid point",
              "bit_identical": same, "all_bit_identical": all(same.values()),
              "resolved": int(np.count_nonzero(np.asarray(got.chip_size)))}
    return cpu, parity, prepared, (ca, cb, cv)


def sample_fields(ar, grid, frac, seed, chip=CHIP):
    n = len(grid)
    idx = np.sort(np.random.default_rng(seed).choice(n, max(1, int(n * frac)), replace=False))
    fl = {f: np.ascontiguousarray(grid.flat(f)[idx]) for f in ar.points.FIELDS}
    fl["chip_size_x"] = np.full(idx.size, chip, np.int64)
    fl["chip_size_y"] = np.full(idx.size, chip, np.int64)
    return idx, fl


def float_flip_rate(ar, ctx, O, ca, cb, cv, seed=3, frac=0.1):
    """Sub-pixel agreement of the unquantised path: the crop highpass-filtered to Float32 (no
    quantisation, so the surfaces carry FP32 products), a seeded sample of the grid at chip
    32 / radius 25 / PyramidRefine(64), the library against the oracle's FP64 numerator. A
    flip is a point whose dx or dy differs by more than 1e-3 px: a near-tie of the 1/64 px
    cascade argmax decided by a last-bit surface difference."""
    p = ar.params(grid_spacing=SPACING, chip_size=CHIP, search_radius=RADIUS, upsampling=UP,
                  quantize="none")
    grid = ar.build_grid(ca.shape, p)
    idx, fl = sample_fields(ar, grid, frac, seed)
    prep = ar.prepare(ar.ImagePair(ca, cb, None, cv), p, ctx)
    ref, sec, rv, sv = prep.download()
    L = ar._lib
    st = L.ArPoints(*(fl[f].ctypes.data for f in ar.points.FIELDS), idx.size)
    g = [np.empty(idx.size, np.float32) for _ in range(3)] + [np.empty(idx.size, np.uint8)]
    ctx.check(ctx.lib.ar_track(ctx.handle, prep.device(ctx).handle, ctypes.byref(st), UP,
                               L.AR_ZNCC, *(x.ctypes.data for x in g)))
    w = O.track(ref, sec, fl, upsampling=UP, reference_valid=rv, secondary_valid=sv)
    m = ~np.isnan(g[0]) & ~np.isnan(w[0])
    d = np.maximum(np.abs(g[0] - w[0]), np.abs(g[1] - w[1]))[m]
    dc = np.abs(g[2] - w[2])[m]
    return {"what": "chip 32 / radius 25 / PyramidRefine(64) on the highpass-filtered Float32 "
                    f"crop ({CROP}^2, quantize = :none), a seeded {int(frac * 100)}% sample, "
                    "library (FP32 products, FP64 sums) against the oracle (FP64 numerator)",
            "points": int(idx.size), "measured_both": int(m.sum()),
            "same_measured_set": bool(np.array_equal(np.isnan(g[0]), np.isnan(w[0]))),
            "flip_rate_over_1e-3px": float(np.mean(d > 1e-3)) if d.size else None,
            "over_half_px": int(np.count_nonzero(d > 0.5)),
            "max_abs_d_px": float(d.max()) if d.size else None,
            "max_abs_dcorr": float(dc.max()) if dc.size else None}


_CV = {}


def _cv_init(ref, sec):
    import cv2
    cv2.setNumThreads(1)
    _CV["ref"], _CV["sec"] = ref, sec


def _cv_points(job):
    """OpenCV's surface, peak and pyrUp cascade at each (row, col) chip centre of `job`
    (0-based, after the +0.5 shift); returns each point's (dx, dy)."""
    import cv2
    ref, sec = _CV["ref"], _CV["sec"]
    h, r = CHIP // 2, RADIUS
    out = np.empty((len(job), 2))
    for k, (y0, x0) in enumerate(job):
        chip = sec[y0 - h:y0 + h, x0 - h:x0 + h]
        win = ref[y0 - h - r:y0 + h + r - 1, x0 - h - r:x0 + h + r - 1]
        s = cv2.matchTemplate(win, chip, cv2.TM_CCOEFF_NORMED)
        i, j = np.unravel_index(int(np.argmax(s)), s.shape)
        i0, j0 = min(max(i - 2, 0), s.shape[0] - 5), min(max(j - 2, 0), s.shape[1] - 5)
        q = np.ascontiguousarray(s[i0:i0 + 5, j0:j0 + 5])
        for _ in range(6):
            q = cv2.pyrUp(q)
        si, sj = np.unravel_index(int(np.argmax(q)), q.shape)
        out[k] = (sj / UP + j0 - r, si / UP + i0 - r)
    return out


def opencv_baseline(ar, grid_fields, prepared):
    """The per-point OpenCV loop (cv2.matchTemplate TM_CCOEFF_NORMED + six cv2.pyrUp steps +
    argmax, the primitives the reference's fixtures come from) on the prepared UInt8 crop at
    chip 32 / radius 25, over every interior grid point of the crop (no padding path), spread
    over the host cores by a pool of spawned worker processes with one OpenCV thread each
    (timed after the pool has started)."""
    try:
        import cv2
    except ImportError:
        return {"unavailable": "OpenCV is not importable"}
    import multiprocessing as mp
    ref = np.ascontiguousarray(prepared[0])
    sec = np.ascontiguousarray(prepared[1])
    nr, nc = ref.shape
    h, r = CHIP // 2, RADIUS
    cy = np.floor(grid_fields["y"] + 0.5).astype(np.int64) - 1  # 0-based
    cx = np.floor(grid_fields["x"] + 0.5).astype(np.int64) - 1
    ok = (cy - h - r >= 0) & (cy + h + r - 1 <= nr) & (cx - h - r >= 0) & (cx + h + r - 1 <= nc)
    centres = np.stack([cy[ok], cx[ok]], axis=1)
    procs = os.cpu_count() or 1
    jobs = np.array_split(centres, max(1, procs * 8))
    with mp.get_context("spawn").Pool(procs, initializer=_cv_init, initargs=(ref, sec)) as pool:
        pool.map(_cv_points, [centres[:1]] * procs)  # workers up and warm
        t0 = time.perf_counter()
        res = pool.map(_cv_points, jobs)
        dt = time.perf_counter() - t0
    done = sum(len(j) for j in jobs)
    return {"value": done / dt, "unit": UNIT, "cores": procs, "kind": "opencv",
            "sample": f"all {done} interior points of the {CROP}^2 crop's grid at chip 32 / "
                      f"radius 25 / x64 (prepared UInt8), {dt:.2f} s; cv2 {cv2.__version__}, "
                      "one process per core, one OpenCV thread each",
            "dxdy": np.concatenate(res) if res else None, "mask": ok}


def opencv_agreement(ar, ctx, cv, cgrid, prepared):
    """The OpenCV loop's offsets against the library's chip-32 pass on the same prepared crop
    and points (OpenCV's FP32 surfaces differ from the exact ones in the last bits, so a few
    1/64 px cascade ties flip)."""
    dxdy, mask = cv.pop("dxdy", None), cv.pop("mask", None)
    if dxdy is None:
        return cv
    fl = {f: np.ascontiguousarray(cgrid.flat(f)[mask]) for f in ar.points.FIELDS}
    fl["chip_size_x"] = np.full(dxdy.shape[0], CHIP, np.int64)
    fl["chip_size_y"] = np.full(dxdy.shape[0], CHIP, np.int64)
    pair = ar.ImagePair(prepared[0], prepared[1], prepared[2], prepared[3])
    L = ar._lib
    st = L.ArPoints(*(fl[f].ctypes.data for f in ar.points.FIELDS), dxdy.shape[0])
    g = [np.empty(dxdy.shape[0], np.float32) for _ in range(3)] + [np.empty(dxdy.shape[0], np.uint8)]
    dp = pair.device(ctx)
    ctx.check(ctx.lib.ar_track(ctx.handle, dp.handle, ctypes.byref(st), UP, L.AR_ZNCC,
                               *(x.ctypes.data for x in g)))
    m = ~np.isnan(g[0])
    d = np.maximum(np.abs(dxdy[:, 0] - g[0]), np.abs(dxdy[:, 1] - g[1]))[m]
    cv["agreement_with_library"] = {"points": int(m.sum()),
                                    "within_1e-3px": float(np.mean(d <= 1e-3)) if d.size else None,
                                    "within_1/32px": float(np.mean(d <= 1 / 32)) if d.size else None}
    return cv


def serving_requests(ar, rng, n_req, sizes, weights, base=None):
    """A mixed request stream in the proportions of the serving configuration: image sides
    `sizes` in the exact relative frequencies `weights` (n_req rounded to a multiple of their
    sum), shuffled; grid spacing from {8, 16, 32}, chip from {16, 32, 64}, search radius
    uniform in [8, 48]. Scenes are generated once per side (host arrays in the column-major
    layout a Julia caller holds)."""
    scenes = {}
    for n in sizes:
        a, b, v = base if (base is not None and base[0].shape[0] == n) else scene(ar, n)
        scenes[n] = (np.asfortranarray(a), np.asfortranarray(b), np.asfortranarray(v))
    k = max(1, int(round(n_req / sum(weights))))
    sides = [n for n, w in zip(sizes, weights) for _ in range(k * w)]
    rng.shuffle(sides)
    reqs = []
    for n in sides:
        kw = dict(grid_spacing=int(rng.choice([8, 16, 32])), chip_size=int(rng.choice([16, 32, 64])),
                  search_radius=int(rng.integers(8, 49)), upsampling=UP)
        reqs.append((int(n), kw))
    return scenes, reqs


def served_e2e(ar, device, ha, hb, hv, hgrid, gr, gc, opts, prm, size, n, pairs, ref_dx,
               slots=3):
    """End to end through the request loop (ar_submit, `slots` slots): `pairs` copies of the
    benchmark pair, each from the caller's host buffers (column-major images, mask and grid),
    submitted together; each is uploaded, prepared, searched and its outputs read back to host
    memory while the others run. Throughput over a whole batch, the median of nine batches after
    two untimed batches that warm every slot (a context's first batches have run up to twice as
    slow on some boxes, and single batches up to three times as slow on a busy host: the copies
    in and out go through host memory the box shares); every result must equal the
    device-resident run's bit for bit."""
    L = ar._lib
    ctx = L.Context(device)
    ctx.set_option(L.AR_OPT_SERVE_SLOTS, slots)
    outs = [[np.empty(n, np.float32) for _ in range(3)] + [np.empty(n, np.uint16),
                                                           np.empty(n, np.uint8)]
            for _ in range(pairs)]

    def batch(k):
        keep, tickets = [], []
        t0 = time.perf_counter()
        for o in outs[:k]:
            req = L.ArRequest(ha.ctypes.data, hb.ctypes.data, None, hv.ctypes.data, size, size,
                              L.AR_U16, opts, prm, ctypes.pointer(hgrid), gr, gc,
                              *(x.ctypes.data for x in o))
            t = L._i64()
            ctx.check(ctx.lib.ar_submit(ctx.handle, ctypes.byref(req), ctypes.byref(t)))
            keep.append(req)
            tickets.append(t.value)
        run = []
        for t in tickets:
            ctx.check(ctx.lib.ar_wait(ctx.handle, t, -1))
            q, r = ctypes.c_double(), ctypes.c_double()
            ctx.check(ctx.lib.ar_request_times(ctx.handle, t, ctypes.byref(q), ctypes.byref(r)))
            run.append(r.value)
            ctx.lib.ar_release(ctx.handle, t)
        return time.perf_counter() - t0, run

    try:
        for _ in range(2):
            batch(pairs)
        timed = [batch(pairs) for _ in range(9)]
        same = all(np.array_equal(o[0].view(np.uint32), ref_dx.view(np.uint32)) for o in outs)
    finally:
        ctx.close()
    rates = [pairs * n / dt for dt, _ in timed]
    return {"value": float(np.median(rates)), "pairs": pairs, "slots": slots,
            "batches_points_per_s": rates,
            "run_ms_p50": float(np.percentile(np.concatenate([r for _, r in timed]), 50)),
            "same_result_as_device_run": bool(same)}


def serving_measure(ar, scenes, reqs, device, slots=4, rates=SERVE_RATES, repeats=2, seed=1):
    """The stream three ways: the plain GPU path (one pair at a time, the direct FP32
    correlation on CUDA cores -- tensor cores off), the same one-pair-at-a-time loop with the
    tensor-core kernels the server runs ("sequential"), and the request loop (continuous
    batching, `slots` slots), alternated `repeats` times after one untimed pass of each
    (medians). Then the request loop under a seeded Poisson stream of the same requests at
    each rate of `rates` (pairs/s): p50/p99 latency from submission to completion (the loop's
    own clock) and the sustained points/s."""
    L = ar._lib
    points = [len(ar.build_grid(scenes[n][0].shape, ar.params(**kw))) for n, kw in reqs]
    plain_ctx = L.Context(device)
    plain_ctx.set_option(L.AR_OPT_TENSOR_CORES, 0)
    seq_ctx = L.Context(device)
    ctx = L.Context(device)
    ctx.set_option(L.AR_OPT_SERVE_SLOTS, slots)

    def one_at_a_time(c):
        out = []
        for n, kw in reqs:
            a, b, v = scenes[n]
            out.append(ar.autorift(a, b, secondary_valid=v, ctx=c, **kw))
        return out

    def served():
        tickets = [ar.submit(*scenes[n][:2], secondary_valid=scenes[n][2], ctx=ctx, **kw)
                   for n, kw in reqs]
        return [t.wait() for t in tickets]

    # Warm-up: the whole stream once through every path (untimed), so every slot has met the
    # largest request and the timed passes see the steady state of a running server.
    plain_res = one_at_a_time(plain_ctx)
    one_at_a_time(seq_ctx)
    served_res = served()
    # Matched accuracy: the served results against the plain path's.
    m = [(~np.isnan(p_.dx)) & (~np.isnan(s_.dx)) for p_, s_ in zip(plain_res, served_res)]
    dd = np.concatenate([np.maximum(np.abs(p_.dx - s_.dx), np.abs(p_.dy - s_.dy))[k]
                         for p_, s_, k in zip(plain_res, served_res, m)])
    del plain_res, served_res
    runs = {"plain": [], "sequential": [], "batched": []}
    for _ in range(repeats):
        for name, fn in (("plain", lambda: one_at_a_time(plain_ctx)),
                         ("sequential", lambda: one_at_a_time(seq_ctx)), ("batched", served)):
            t0 = time.perf_counter()
            fn()
            runs[name].append(time.perf_counter() - t0)
    plain_ctx.close()
    seq_ctx.close()
    med = {k: float(np.median(v)) for k, v in runs.items()}
    cap = len(reqs) / med["batched"]
    total = float(sum(points))
    sweep = []
    for i, rate in enumerate(rates):
        rng = np.random.default_rng(seed + i)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
        t0 = time.perf_counter()
        tickets = []
        for (n, kw), at in zip(reqs, arrivals):
            dt = at - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            tickets.append(ar.submit(*scenes[n][:2], secondary_valid=scenes[n][2], ctx=ctx, **kw))
        lat, big = [], []
        for (n, _), t in zip(reqs, tickets):
            t.wait()
            q, r = t.times()
            lat.append(q + r)
            if n == max(scenes):
                big.append(q + r)
        stream_s = time.perf_counter() - t0
        del tickets
        sweep.append({"rate_pairs_per_s": rate, "p50_ms": float(np.percentile(lat, 50)),
                      "p99_ms": float(np.percentile(lat, 99)),
                      "largest_pairs_p50_ms": float(np.percentile(big, 50)) if big else None,
                      "points_per_s": total / stream_s, "seconds": stream_s})
    ctx.close()
    counts = {str(n): sum(1 for m_, _ in reqs if m_ == n) for n in sorted(scenes)}
    return {"requests": len(reqs), "requests_per_side": counts, "points": int(total),
            "slots": slots, "repeats": repeats,
            "plain_points_per_s": total / med["plain"],
            "plain_path": "one pair at a time, direct FP32 correlation on CUDA cores "
                          "(AR_OPT_TENSOR_CORES = 0)",
            "sequential_points_per_s": total / med["sequential"],
            "batched_points_per_s": total / med["batched"], "batched_pairs_per_s": cap,
            "speedup_vs_plain": med["plain"] / med["batched"],
            "speedup_per_repeat": [p_ / q_ for p_, q_ in zip(runs["plain"], runs["batched"])],
            "speedup_vs_sequential": med["sequential"] / med["batched"],
            "matched_accuracy": {"points_compared": int(dd.size),
                                 "dx_dy_within_1e-3px": float(np.mean(dd <= 1e-3))
                                 if dd.size else None},
            "sweep": sweep}


def oracle_sample(ar, ctx, raw, opts, grid, size, seed=1):
    """The oracle on a seeded 1% sample of the step's points: the chip-32 pass (radius 25,
    PyramidRefine(64), ZNCC) on the prepared pair, the library against the oracle's FP64
    numerator on the same points and inputs."""
    from oracle import oracle as O
    L = ar._lib
    lib = ctx.lib
    O.build()
    prep = ctypes.c_void_p()
    ctx.check(lib.ar_prepare(ctx.handle, raw.handle, ctypes.byref(opts), ctypes.byref(prep)))
    try:
        ref, sec = (np.empty((size, size), np.uint8, order="F") for _ in range(2))
        rv, sv = (np.empty((size, size), np.uint8, order="F") for _ in range(2))
        ctx.check(lib.ar_pair_download(ctx.handle, prep, ref.ctypes.data, sec.ctypes.data,
                                       rv.ctypes.data, sv.ctypes.data))
        n = len(grid)
        idx = np.sort(np.random.default_rng(seed).choice(n, n // 100, replace=False))
        fl = {f: np.ascontiguousarray(grid.flat(f)[idx]) for f in ar.points.FIELDS}
        fl["chip_size_x"] = np.full(idx.size, CHIP, np.int64)
        fl["chip_size_y"] = np.full(idx.size, CHIP, np.int64)
        st = L.ArPoints(*(fl[f].ctypes.data for f in ar.points.FIELDS), idx.size)
        g = [np.empty(idx.size, np.float32) for _ in range(3)] + [np.empty(idx.size, np.uint8)]
        ctx.check(lib.ar_track(ctx.handle, prep, ctypes.byref(st), UP, L.AR_ZNCC,
                               *(a.ctypes.data for a in g)))
        w = O.track(ref, sec, fl, upsampling=UP, reference_valid=rv, secondary_valid=sv)
    finally:
        lib.ar_pair_destroy(prep)
    same = [bool(np.array_equal(a.view(np.uint32), b.view(np.uint32))) for a, b in zip(g[:3], w[:3])]
    return {"points": int(idx.size), "seed": seed,
            "pass": f"chip {CHIP}, radius {RADIUS}, PyramidRefine({UP}) on the prepared pair",
            "dx_dy_correlation_bit_identical": all(same),
            "searched_identical": bool(np.array_equal(g[3].astype(bool), w[3])),
            "measured": int(np.count_nonzero(~np.isnan(w[0])))}


ROT_ANGLES = (-3.0, 0.0, 3.0)  # RotationSearch()'s default, src/types.jl:557


def rotation_measure(ar, ctx, raw, opts, grid, args, dev, stream, flush, fp32_peak, rank, world,
                     size):
    """The rotation search (src/track.jl:313-409) over the fine level's point set: every grid
    point at chip 32 / radius 25 with RotationSearch() (angles -3, 0, 3), on the prepared pair,
    PyramidRefine(64). Device-timed like the main step, beside the same pass without rotation,
    and the oracle's restatement timed on a sample of the same points."""
    import torch
    L = ar._lib
    lib = ctx.lib
    prep = ctypes.c_void_p()
    ctx.check(lib.ar_prepare(ctx.handle, raw.handle, ctypes.byref(opts), ctypes.byref(prep)))
    n = len(grid)
    cols = {f: torch.from_numpy(grid.flat(f)).to(dev) for f in ar.points.FIELDS}
    cols["chip_size_x"].fill_(CHIP)
    cols["chip_size_y"].fill_(CHIP)
    pts = L.ArPoints(*(cols[f].data_ptr() for f in ar.points.FIELDS), n)
    outs = [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3)]
    osr = torch.empty(n, dtype=torch.uint8, device=dev)
    angs = np.asarray(ROT_ANGLES, dtype=np.float64)
    res = {}
    steps = max(3, args.steps // 4)
    try:
        for name, count in (("rotation", angs.size), ("plain", 0)):
            def call():
                ctx.check(lib.ar_track_device_rotated(
                    ctx.handle, prep, ctypes.byref(pts), UP, L.AR_ZNCC, angs.ctypes.data, count,
                    outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), osr.data_ptr(),
                    None))
            with torch.cuda.stream(stream):
                for _ in range(args.warmup):
                    flush.fill_(1)
                    call()
                torch.cuda.synchronize()
                ctx.set_timing(True)
                ctx.kernel_times()
                tot = 0.0
                for _ in range(steps):
                    flush.fill_(1)
                    ev0 = torch.cuda.Event(enable_timing=True)
                    ev1 = torch.cuda.Event(enable_timing=True)
                    ev0.record(stream)
                    call()
                    ev1.record(stream)
                    ev1.synchronize()
                    tot += ev0.elapsed_time(ev1)
                corr_ms, refine_ms, _, launches, flops = ctx.kernel_times()
                ctx.set_timing(False)
            res[name] = {"points_per_s": world * n * steps / (tot * 1e-3),
                         "ms_per_pass": tot / steps, "k_corr_ms": corr_ms / steps,
                         "k_refine_ms": refine_ms / steps,
                         "corr_tflops": flops / (corr_ms * 1e-3) / 1e12 if corr_ms > 0 else None,
                         "launches_per_pass": launches / steps}
        rot_dx = outs[0].cpu().numpy()
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            from oracle import oracle as O
            O.build()
            ref, sec = (np.empty((size, size), np.uint8, order="F") for _ in range(2))
            rv, sv = (np.empty((size, size), np.uint8, order="F") for _ in range(2))
            ctx.check(lib.ar_pair_download(ctx.handle, prep, ref.ctypes.data, sec.ctypes.data,
                                           rv.ctypes.data, sv.ctypes.data))
            idx = np.linspace(0, n - 1, 10000).astype(np.int64)
            fl = {f: grid.flat(f)[idx] for f in ar.points.FIELDS}
            fl["chip_size_x"] = np.full(idx.size, CHIP, np.int64)
            fl["chip_size_y"] = np.full(idx.size, CHIP, np.int64)
            t0 = time.perf_counter()
            wdx = O.track(ref, sec, fl, upsampling=UP, reference_valid=rv, secondary_valid=sv,
                          angles=ROT_ANGLES)[0]
            dt = time.perf_counter() - t0
            m = ~np.isnan(wdx) & ~np.isnan(rot_dx[idx])
            cpu = {"value": idx.size / dt, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
                   "sample": f"{idx.size} of the {n} points (evenly spaced), three angles, "
                             f"{dt:.1f} s",
                   "dx_agree_1e-3px": float(np.mean(np.abs(wdx[m] - rot_dx[idx][m]) <= 1e-3))
                   if m.any() else None}
    finally:
        lib.ar_pair_destroy(prep)
    r = res["rotation"]
    return {"workload": f"track over the {n} grid points at chip {CHIP}, radius {RADIUS}, "
                        f"PyramidRefine({UP}), RotationSearch() angles {list(ROT_ANGLES)}, on the "
                        "prepared UInt8 pair; L2 flushed before each pass",
            "points_per_s": r["points_per_s"], "ms_per_pass": r["ms_per_pass"],
            "kernel_ms_per_pass": {"k_corr": r["k_corr_ms"], "k_refine": r["k_refine_ms"]},
            "plain_points_per_s": res["plain"]["points_per_s"],
            "cost_vs_plain": res["plain"]["points_per_s"] / r["points_per_s"],
            "roofline": {"bound": "fp32", "kernel": "k_corr (rotation instantiation)",
                         "achieved": r["corr_tflops"], "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": r["corr_tflops"] / fp32_peak if (r["corr_tflops"] and fp32_peak)
                         else None,
                         "peak_source": "cuBLAS SGEMM (TF32 off) measured in this run",
                         "achieved_basis": "2 * chip area * surface area per point and angle"},
            "cpu_baseline": cpu, "gpu_launches_per_pass": r["launches_per_pass"]}


class DeviceStep:
    """One step of the pipeline on a device-resident raw pair and grid: ar_prepare, then
    ar_multichip_device, on the context's stream."""

    def __init__(self, ar, ctx, torch, dev, a, b, valid, p, grid=None):
        L = ar._lib
        self.ctx, self.lib = ctx, ctx.lib
        self.grid = grid if grid is not None else ar.build_grid(a.shape, p)
        self.gr, self.gc = self.grid.shape
        self.n = self.gr * self.gc
        self.raw = ar.ImagePair(a, b, None, valid).device(ctx)  # resident before timing
        self.cols = {f: torch.from_numpy(self.grid.flat(f)).to(dev) for f in ar.points.FIELDS}
        self.dgrid = L.ArPoints(*(self.cols[f].data_ptr() for f in ar.points.FIELDS), self.n)
        self.outs = [torch.empty(self.n, dtype=torch.float32, device=dev) for _ in range(3)]
        self.ochip = torch.empty(self.n, dtype=torch.int16, device=dev)
        self.oint = torch.empty(self.n, dtype=torch.uint8, device=dev)
        self.prm = ar.multichip_params(p)
        self.opts = ar.prepare_options(p)

    def __call__(self):
        ctx, lib = self.ctx, self.lib
        prep = ctypes.c_void_p()
        ctx.check(lib.ar_prepare(ctx.handle, self.raw.handle, ctypes.byref(self.opts),
                                 ctypes.byref(prep)))
        try:
            ctx.check(lib.ar_multichip_device(
                ctx.handle, prep, ctypes.byref(self.dgrid), self.gr, self.gc,
                ctypes.byref(self.prm), self.outs[0].data_ptr(), self.outs[1].data_ptr(),
                self.outs[2].data_ptr(), self.ochip.data_ptr(), self.oint.data_ptr(), None))
        finally:
            lib.ar_pair_destroy(prep)


def timed_steps(torch, step, stream, flush, steps, warmup, dist=None):
    """Device time (ms, summed over `steps`) of `step`, CUDA events on the library's stream,
    L2 flushed before every step (outside the timed interval)."""
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            flush.fill_(1)
            step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        total = 0.0
        for _ in range(steps):
            flush.fill_(1)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            step()
            e.record(stream)
            e.synchronize()
            total += s.elapsed_time(e)
        torch.cuda.synchronize()
    return total


def host_e2e(ar, ctx, hostpair, hgrid, gr, gc, opts, prm, size, n, reps):
    """One pair at a time through the C ABI from host buffers: ar_pair_upload + ar_prepare +
    ar_multichip (results read back to host memory); seconds per pair, the outputs of the last."""
    L, lib = ar._lib, ctx.lib
    ha, hb, hv = hostpair
    hout = [np.empty(n, np.float32) for _ in range(3)]
    hchip = np.empty(n, np.uint16)
    hint = np.empty(n, np.uint8)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        rp, pp = ctypes.c_void_p(), ctypes.c_void_p()
        ctx.check(lib.ar_pair_upload(ctx.handle, ha.ctypes.data, hb.ctypes.data, None,
                                     hv.ctypes.data, size, size, L.AR_U16, ctypes.byref(rp)))
        ctx.check(lib.ar_prepare(ctx.handle, rp, ctypes.byref(opts), ctypes.byref(pp)))
        ctx.check(lib.ar_multichip(ctx.handle, pp, ctypes.byref(hgrid), gr, gc, ctypes.byref(prm),
                                   hout[0].ctypes.data, hout[1].ctypes.data, hout[2].ctypes.data,
                                   hchip.ctypes.data, hint.ctypes.data))
        lib.ar_pair_destroy(pp)
        lib.ar_pair_destroy(rp)
        times.append(time.perf_counter() - t0)
    return times, hout, hchip


def batching_measure(ar, ctx, torch, dev, a, b, valid, fdown, stream, flush, args):
    """The batching configuration on the benchmark pair: chip sizes 16/32/64/128 through the
    multichip search over ~1.9 M jittered centres on an 8 px lattice with per-point radii
    U[4, 48] (floored to 6 by sanitize!) and integer priors from the 4x-downsampled imposed
    field +-3 px. Timed two ways on the device -- shape-binned passes with the autotuned kernel
    choice (the default) and one launch per pass planned for its largest surface with the
    default kernel rule -- with bit-identical results required."""
    L = ar._lib
    n = a.shape[0]
    X, Y, r, dx0, dy0 = ar.synthetic.batching_points(n, fdown[0], fdown[1])
    grid = ar.pointset(X, Y, search_radius_x=r, search_radius_y=r, chip_size=128,
                       dx_prior=dx0, dy_prior=dy0)
    p = ar.params(chip_size=16, chip_size_max=128, upsampling=UP)
    step = DeviceStep(ar, ctx, torch, dev, a, b, valid, p, grid=grid)
    out = {}
    res = {}
    steps = max(3, args.steps // 4)
    for name, bins, tune in (("binned_autotuned", 1, 1), ("one_launch_per_pass", 0, 0)):
        ctx.set_option(L.AR_OPT_SHAPE_BINS, bins)
        ctx.set_option(L.AR_OPT_AUTOTUNE, tune)
        t = timed_steps(torch, step, stream, flush, steps, args.warmup)
        out[name] = {"points_per_s": step.n * steps / (t * 1e-3), "ms_per_step": t / steps}
        res[name] = [o.cpu().numpy() for o in step.outs] + [step.ochip.cpu().numpy()]
    ctx.set_option(L.AR_OPT_SHAPE_BINS, 1)
    ctx.set_option(L.AR_OPT_AUTOTUNE, 1)
    same = all(np.array_equal(x.view(np.uint32) if x.dtype == np.float32 else x,
                              y.view(np.uint32) if y.dtype == np.float32 else y)
               for x, y in zip(res["binned_autotuned"], res["one_launch_per_pass"]))
    chip = res["binned_autotuned"][3].view(np.uint16)
    out.update({"points": step.n, "grid": list(step.grid.shape), "steps": steps,
                "speedup": out["one_launch_per_pass"]["ms_per_step"] /
                           out["binned_autotuned"]["ms_per_step"],
                "bit_identical": bool(same),
                "points_per_chip_size": {int(c): int(np.count_nonzero(chip == c))
                                         for c in np.unique(chip) if c},
                "workload": f"multichip 16/32/64/128 on the {n}^2 benchmark pair, jittered 8 px "
                            "lattice, radii U[4,48], priors from the 4x-downsampled field +-3 px "
                            "(the benchmark scene's 15 px bumps: the 40 px scene of the "
                            "batching configuration would add another scene generation to "
                            "the run), PyramidRefine(64)"})
    return out


def bf16_executed_flops(ch, cw, nr, products=6):
    """Tensor-core FLOPs k_corr_bf executes for one point: per 16-row window block the products
    of M = 64 surface columns, the block's trimmed operand rows and K = 16, for every chip
    column and limb pair (six for Float32 imagery, five for integer imagery)."""
    NB = (ch + 15 + 15) // 16 * 16
    QB = (ch + nr - 1 + 15) // 16
    rows = 0
    for q in range(QB):
        lo = max(0, NB - 16 - 16 * q)
        hi = min(NB, NB - 16 + nr - 16 * q)
        if hi > lo:
            elo = lo & ~15
            rows += (hi - elo + 15) & ~15
    return 2.0 * 64 * 16 * rows * cw * products


def precision_measure(ar, ctx, torch, dev, a4, b4, v4, fdown4, stream, flush, args, tensor_peak):
    """The precision configuration on the 4096^2 pair: the default pipeline restricted to chip
    sizes 64 and 128 at search radius 32, unquantised (highpass Float32), its correlation
    numerators computed three ways -- split BF16 on the tensor cores, direct FP32 on CUDA cores
    (AR_OPT_SPLIT_BF16 = 1 / 0) and the oracle's FP64 -- on a seeded sample of each grid:
    max |dNCC|, integer-peak agreement (integer offsets identical), sub-pixel |dd|, and the
    error against the imposed field; plus each variant's device-timed pass over the whole grid
    and the split-BF16 kernel's rate against the tensor-pipe peak."""
    from oracle import oracle as O
    L = ar._lib
    O.build()
    out = {"workload": "chip 64 and 128, radius 32, highpass Float32 (quantize = :none) on the "
                       "4096^2 benchmark pair: one track pass over the spacing-8 grid per chip "
                       "size; the oracle on a seeded sample (0.5% at chip 64, 0.25% at 128)"}
    fx_d, fy_d = fdown4
    for chip in (64, 128):
        p = ar.params(chip_size=chip, search_radius=32, quantize="none", upsampling=UP)
        grid = ar.gridpoints(a4.shape, 8, chip_size=chip, search_radius=32)
        n = len(grid)
        cols = {f: torch.from_numpy(grid.flat(f)).to(dev) for f in ar.points.FIELDS}
        pts = L.ArPoints(*(cols[f].data_ptr() for f in ar.points.FIELDS), n)
        outs = [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3)]
        srch = torch.empty(n, dtype=torch.uint8, device=dev)
        # The oracle's FP64 numerator costs 2 chip area x surface area per point per pass:
        # a 0.5% sample at chip 64, 0.25% at chip 128.
        idx, fl = sample_fields(ar, grid, 0.005 if chip == 64 else 0.0025, seed=7, chip=chip)
        row = {"points": n}
        want = None
        for name, mode in (("split_bf16", 1), ("direct_fp32", 0)):
            ctx.set_option(L.AR_OPT_SPLIT_BF16, mode)
            prep = ar.prepare(ar.ImagePair(a4, b4, None, v4), p, ctx)
            h = prep.device(ctx).handle

            def call():
                ctx.check(ctx.lib.ar_track_device(ctx.handle, h, ctypes.byref(pts), UP, L.AR_ZNCC,
                                                  outs[0].data_ptr(), outs[1].data_ptr(),
                                                  outs[2].data_ptr(), srch.data_ptr(), None))
            timed_steps(torch, call, stream, flush, 0, 1)
            ctx.set_timing(True)
            ctx.kernel_times()
            t = timed_steps(torch, call, stream, flush, 2, 0)
            corr_ms, refine_ms, tracks, _, flops = ctx.kernel_times()
            ctx.set_timing(False)
            dx = outs[0].cpu().numpy()
            r = {"points_per_s": 2 * n / (t * 1e-3), "k_corr_ms": corr_ms / 2,
                 "k_refine_ms": refine_ms / 2,
                 "algorithmic_tflops": flops / (corr_ms * 1e-3) / 1e12 if corr_ms > 0 else None}
            if mode == 1 and corr_ms > 0:
                executed = bf16_executed_flops(chip, chip, 64) * (flops / (2.0 * chip * chip * 64 * 64))
                r["executed_tensor_tflops"] = executed / (corr_ms * 1e-3) / 1e12
                r["frac_of_bf16_peak"] = r["executed_tensor_tflops"] / tensor_peak
            # Accuracy on the sample, against the oracle (FP64 numerator) and the imposed field.
            st = L.ArPoints(*(fl[f].ctypes.data for f in ar.points.FIELDS), idx.size)
            g = [np.empty(idx.size, np.float32) for _ in range(3)] + [np.empty(idx.size, np.uint8)]
            ctx.check(ctx.lib.ar_track(ctx.handle, h, ctypes.byref(st), UP, L.AR_ZNCC,
                                       *(x.ctypes.data for x in g)))
            if want is None:
                ref, sec, rv, sv = prep.download()
                want = O.track(ref, sec, fl, upsampling=UP, reference_valid=rv, secondary_valid=sv)
                wi = O.track(ref, sec, fl, upsampling=1, reference_valid=rv, secondary_valid=sv)
            gi = [np.empty(idx.size, np.float32) for _ in range(3)] + [np.empty(idx.size, np.uint8)]
            ctx.check(ctx.lib.ar_track(ctx.handle, h, ctypes.byref(st), 1, L.AR_ZNCC,
                                       *(x.ctypes.data for x in gi)))
            m = ~np.isnan(g[0]) & ~np.isnan(want[0])
            d = np.maximum(np.abs(g[0] - want[0]), np.abs(g[1] - want[1]))[m]
            mi = ~np.isnan(gi[0]) & ~np.isnan(wi[0])
            same_int = (gi[0][mi] == wi[0][mi]) & (gi[1][mi] == wi[1][mi])
            iy = np.clip(np.round(fl["y"] - 1).astype(int) // 4, 0, fx_d.shape[0] - 1)
            ix = np.clip(np.round(fl["x"] - 1).astype(int) // 4, 0, fx_d.shape[1] - 1)
            fe = np.hypot(g[0] + fx_d[iy, ix], g[1] + fy_d[iy, ix])[~np.isnan(g[0])]
            r.update({"sample_points": int(idx.size), "measured": int(m.sum()),
                      "max_abs_dncc": float(np.abs(g[2] - want[2])[m].max()) if m.any() else None,
                      "integer_peak_agreement": float(same_int.mean()) if mi.any() else None,
                      "subpixel_max_abs_dd_px": float(d.max()) if d.size else None,
                      "subpixel_over_1e-3px": float(np.mean(d > 1e-3)) if d.size else None,
                      "median_error_vs_field_px": float(np.median(fe)) if fe.size else None})
            row[name] = r
            del prep
        ctx.set_option(L.AR_OPT_SPLIT_BF16, 1)
        out[f"chip_{chip}"] = row
    return out


def gpu_arm(args):
    import torch
    import __graft_entry__ as ge

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    ge.build()
    ar = ge.load_package()
    L = ar._lib
    ctx = L.Context(local)
    if args.profile:
        # Under a profiler every launch is serialised and cold, which distorts the autotuner's
        # timing of its samples (under ncu it kept k_corr_tc for the fine pass, which the
        # timed run does not): profile runs take the fixed rule, which picks the kernels the
        # tuned run keeps on this workload (k_corr_tc2 up to chip 64, k_corr_tc at chip 128).
        ctx.set_option(L.AR_OPT_AUTOTUNE, 0)
    a, b, valid, fdown = scene(ar, args.size, field=True)
    p = pipeline_params(ar, args.spacing if args.profile else SPACING)
    dev = torch.device("cuda", local)
    step = DeviceStep(ar, ctx, torch, dev, a, b, valid, p)
    grid, gr, gc, n = step.grid, step.gr, step.gc, step.n
    raw, opts, prm = step.raw, step.opts, step.prm
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    torch.cuda.synchronize()

    timed_steps(torch, step, stream, flush, 0, args.warmup, dist)
    ctx.set_timing(True)
    ctx.kernel_times()
    with ClockSampler(local) as clk:
        total_ms = timed_steps(torch, step, stream, flush, args.steps, 0, dist)
    corr_ms, refine_ms, tracks, launches, corr_flops = ctx.kernel_times()
    ctx.set_timing(False)
    if dist:
        dist.barrier()
    total_ms, value = replicas_rate(dist, total_ms, n, args.steps, dev)
    ms_per_step = total_ms / args.steps

    dx = step.outs[0].cpu().numpy()
    chip = step.ochip.cpu().numpy().view(np.uint16)
    resolved = int(np.count_nonzero(chip))
    achieved = corr_flops / (corr_ms * 1e-3) / 1e12 if corr_ms > 0 else None
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_run": True, "points": n, "ms_per_step": ms_per_step,
                              "k_corr_ms": corr_ms / args.steps,
                              "k_refine_ms": refine_ms / args.steps}))
        if dist:
            dist.destroy_process_group()
        return

    # The plain GPU path on the same step: the direct FP32 correlation on CUDA cores (tensor
    # cores off), one pair at a time, timed the same way; and its agreement with the results
    # above (both numerators are exact for UInt8, so dx agrees to the bit).
    ctx.set_option(L.AR_OPT_TENSOR_CORES, 0)
    psteps = 3
    ptot = timed_steps(torch, step, stream, flush, psteps, 1, dist)
    ctx.set_option(L.AR_OPT_TENSOR_CORES, 1)
    ptot, prate = replicas_rate(dist, ptot, n, psteps, dev)
    pdx = step.outs[0].cpu().numpy()
    plain = {"points_per_s": prate, "ms_per_step": ptot / psteps, "steps": psteps,
             "path": "the same step with AR_OPT_TENSOR_CORES = 0: the direct FP32 "
                     "correlation on CUDA cores (k_corr), one pair at a time",
             "speedup": value / prate,
             "identical_dx": bool(np.array_equal(pdx.view(np.uint32), dx.view(np.uint32)))}
    levels = {int(c): int(np.count_nonzero(chip == c)) for c in np.unique(chip) if c}
    med_dx = float(np.nanmedian(dx)) if resolved else float("nan")

    fp32_peak = measure_fp32_peak(torch, dev)
    eval_flops = 2.0 * CHIP * CHIP * (2 * RADIUS) ** 2
    fine_points = corr_flops / max(tracks, 1) / eval_flops  # chip-32 evaluations per launch
    tuned_kernels = ctx.tuned()
    fine_kernel = fine_pass_kernel(ctx)

    # End to end through the C ABI from host buffers: the caller's column-major arrays (the
    # Julia layout) and grid, pair upload, prepare, multichip, download; per-pair latency.
    hostpair = (np.asfortranarray(a), np.asfortranarray(b),
                np.asfortranarray(valid.astype(np.uint8)))
    hcols = {f: np.ascontiguousarray(grid.flat(f)) for f in ar.points.FIELDS}
    hgrid = L.ArPoints(*(hcols[f].ctypes.data for f in ar.points.FIELDS), n)
    e2e_times, hout, hchip = host_e2e(ar, ctx, hostpair, hgrid, gr, gc, opts, prm, args.size, n,
                                      args.warmup + min(args.steps, 10))
    e2e_times = e2e_times[args.warmup:]
    e2e_value = world * n / float(np.mean(e2e_times))
    same = bool(np.array_equal(hchip, chip)) and bool(
        np.array_equal(hout[0].view(np.uint32), dx.view(np.uint32)))
    # The plain path end to end, one pair at a time from host buffers (tensor cores off).
    ctx.set_option(L.AR_OPT_TENSOR_CORES, 0)
    pe_times, _, _ = host_e2e(ar, ctx, hostpair, hgrid, gr, gc, opts, prm, args.size, n, 3)
    ctx.set_option(L.AR_OPT_TENSOR_CORES, 1)
    plain_e2e = world * n / float(np.mean(pe_times[1:]))
    served = served_e2e(ar, local, *hostpair, hgrid, gr, gc, opts, prm, args.size, n,
                        pairs=min(args.steps, 12), ref_dx=dx)
    h2d = sum(x.nbytes for x in hostpair) + 6 * 8 * n
    d2h = n * (4 + 4 + 4 + 2 + 1)

    parity = cpu = crop_check = flips = cv = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        try:
            parity = oracle_sample(ar, ctx, raw, opts, grid, args.size)
        except Exception as exc:  # reported, not fatal to the main measurement
            parity = {"error": f"{type(exc).__name__}: {exc}"}
        try:
            cpu, crop_check, prepared, cropped = crop_parity(ar, ctx, O, a, b, valid, p)
            flips = float_flip_rate(ar, ctx, O, *cropped)
            cgrid = ar.build_grid(cropped[0].shape, p)
            cv = opencv_baseline(ar, {f: cgrid.flat(f) for f in ("x", "y")}, prepared)
            cv = opencv_agreement(ar, ctx, cv, cgrid, prepared)
        except Exception as exc:
            crop_check = {"error": f"{type(exc).__name__}: {exc}"}
        if world > 1:
            cpu = None  # the host baseline is a single-process figure

    # The at-scale configuration's 4096^2 pair, timed the same way (device-resident).
    a4, b4, v4, fdown4 = scene(ar, N_SCALE, field=True)
    step4 = DeviceStep(ar, ctx, torch, dev, a4, b4, v4, p)
    t4 = timed_steps(torch, step4, stream, flush, args.steps, args.warmup, dist)
    t4, v4rate = replicas_rate(dist, t4, step4.n, args.steps, dev)
    config_4096 = {"workload": workload(N_SCALE, step4.gr, step4.gc), "points": step4.n,
                   "value": v4rate, "ms_per_step": t4 / args.steps}

    peaks = measured_peaks()
    tensor_peak = float(peaks["bf16_tflops"]) if peaks.get("bf16_tflops") else 1590.0
    precision = None
    if rank == 0:
        try:
            precision = precision_measure(ar, ctx, torch, dev, a4, b4, v4, fdown4, stream, flush,
                                          args, tensor_peak)
        except Exception as exc:  # reported, not fatal to the main measurement
            precision = {"error": f"{type(exc).__name__}: {exc}"}

    batching = None
    if not args.profile:
        try:
            batching = batching_measure(ar, ctx, torch, dev, a, b, valid, fdown, stream, flush,
                                        args)
        except Exception as exc:  # reported, not fatal to the main measurement
            batching = {"error": f"{type(exc).__name__}: {exc}"}

    rotation = None
    if not args.no_rotation:
        try:
            rotation = rotation_measure(ar, ctx, step4.raw, opts, step4.grid, args, dev, stream,
                                        flush, fp32_peak, rank, world, N_SCALE)
        except Exception as exc:  # reported, not fatal to the main measurement
            rotation = {"error": f"{type(exc).__name__}: {exc}"}
    del step4

    serving = None
    if not args.no_serving:
        # The serving configuration's mixed stream (sides 512, 2048, 4096, 10980 in 8:4:2:1)
        # through the plain path, the sequential path and the request loop, then the Poisson
        # sweep.
        try:
            sc, reqs = serving_requests(ar, np.random.default_rng(5), 30,
                                        (512, 2048, N_SCALE, N), (8, 4, 2, 1),
                                        base=(a, b, valid))
            serving = serving_measure(ar, sc, reqs, local)
            serving["workload"] = (
                f"{len(reqs)} requests, sides 512/2048/4096/10980 (8:4:2:1), spacing "
                "{8,16,32}, chip {16,32,64}, radius U[8,48], PyramidRefine(64); after one "
                "untimed pass of the stream through every path, plain, sequential and batched "
                "passes alternated (medians); then the same requests as a seeded Poisson "
                f"stream at each of {list(SERVE_RATES)} pairs/s: latency from submission to "
                "completion")
        except Exception as exc:  # reported, not fatal to the main measurement
            serving = {"error": f"{type(exc).__name__}: {exc}"}

    peaks = measured_peaks()
    if peaks.get("bf16_tflops"):
        tensor_peak = float(peaks["bf16_tflops"])
        peak_source = ("MEASURED_PEAKS.json bf16_tflops (burst cuBLAS bf16 GEMM; each "
                       "correlation launch is timed on its own); of measured")
    else:
        tensor_peak = 1590.0
        peak_source = "fallback 1.59 PFLOP/s bf16 (no MEASURED_PEAKS.json); of fallback"
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic",
            "config": {"workload": workload(args.size, gr, gc), "points": n, "grid": [gr, gc],
                       "resolved": resolved, "points_per_chip_size": levels,
                       "chip": CHIP, "radius": RADIUS, "upsampling": UP,
                       "image": [args.size, args.size], "element_type": "uint16 -> uint8",
                       "masks": "secondary no-data mask passed",
                       "l2": "flushed (256 MiB write) between steps",
                       "parallelism": f"{world} independent replicas", "median_dx": med_dx},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": tensor_peak,
                         "unit": "TFLOP/s",
                         "frac": achieved / tensor_peak if achieved else None,
                         "traffic": profile_traffic(fine_points, fine_kernel),
                         "kernel": fine_kernel, "tuned_kernels": tuned_kernels,
                         "peak_source": peak_source,
                         "achieved_basis": "2 * chip area * surface area per searched point "
                                           "(integer MACs of the exact u8 numerator), summed "
                                           "over the step's correlation launches",
                         "frac_of_int8_rate": achieved / (2 * tensor_peak) if achieved else None,
                         "int8_rate_note": "the products are tcgen05.mma kind::i8, whose dense "
                                           "rate is twice the bf16 rate: frac_of_int8_rate "
                                           "divides by 2 x peak",
                         "fp32_comparison": {"sgemm_tflops_this_run": fp32_peak,
                                             "frac": achieved / fp32_peak
                                             if (achieved and fp32_peak) else None},
                         "kernel_ms_per_step": {"k_corr": corr_ms / args.steps,
                                                "k_refine": refine_ms / args.steps},
                         "correlation_launches_per_step": tracks / args.steps,
                         "measured_peaks": {k: peaks.get(k) for k in ("hbm_gbs", "bf16_tflops")}},
            "cpu_baseline": cpu,
            "cpu_baseline_opencv": cv,
            "e2e": {"value": world * served["value"], "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "path": f"ar_submit request loop, {served['slots']} slots: "
                            f"{served['pairs']} pairs from host buffers submitted together, "
                            "each uploaded, prepared, searched and read back (median of 9 "
                            "batches)",
                    "batches_points_per_s": served["batches_points_per_s"],
                    "p50_ms": float(np.percentile(e2e_times, 50)) * 1e3,
                    "p99_ms": float(np.percentile(e2e_times, 99)) * 1e3,
                    "latency": "p50/p99 of one pair alone (one_pair_at_a_time below)",
                    "served_run_ms_p50": served["run_ms_p50"],
                    "same_result_as_device_run": same and served["same_result_as_device_run"],
                    "one_pair_at_a_time": {
                        "value": e2e_value,
                        "path": "ar_pair_upload + ar_prepare + ar_multichip (host buffers), "
                                "one pair after another"}},
            "plain_gpu_path": plain,
            "batched_vs_plain": {
                "served_e2e_points_per_s": world * served["value"],
                "plain_e2e_points_per_s": plain_e2e,
                "ratio_e2e": world * served["value"] / plain_e2e,
                "ratio_device": value / prate, "target": 3.0,
                "plain_e2e_path": "ar_pair_upload + ar_prepare + ar_multichip from host "
                                  "buffers with AR_OPT_TENSOR_CORES = 0, one pair at a time "
                                  "(mean of 2 after 1 warm-up)"},
            "oracle_sample": parity,
            "oracle_crop": crop_check,
            "float32_subpixel": flips,
            "config_4096": config_4096,
            "batching": batching,
            "precision": precision,
            "serving": serving,
            "rotation_search": rotation,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def profile_pass_arm(args, precision):
    """For ncu captures of one correlation pass: a single track pass over the --size pair at grid
    spacing --spacing, `--warmup` untimed passes then `--steps` timed ones; prints one line of
    timings. precision: the split-BF16 kernel's chip-64 / radius-32 pass on the highpass-filtered
    Float32 pair (quantize = :none); otherwise the fine chip-32 / radius-25 pass of the default
    pipeline on the prepared UInt8 pair with the autotuner off (k_corr_tc2). --chip / --radius
    replace the pass's chip size and radius (a radius above 32 runs k_corr_tc); --kernel picks
    the UInt8 kernel."""
    import torch
    import __graft_entry__ as ge

    ge.build()
    ar = ge.load_package()
    L = ar._lib
    ctx = L.Context(0)
    a, b, v = scene(ar, args.size)
    chip, radius = (64, 32) if precision else (32, 25)
    chip = args.chip or chip
    radius = args.radius or radius
    if precision:
        p = ar.params(chip_size=chip, search_radius=radius, quantize="none", upsampling=UP)
    else:
        p = ar.params(chip_size=chip, search_radius=radius, upsampling=UP)
        ctx.set_option(L.AR_OPT_AUTOTUNE, 0)
        if args.kernel:
            ctx.set_option(L.AR_OPT_UINT8_KERNEL, {"tc2": 2, "tc": 1, "direct": 0}[args.kernel])
    grid = ar.gridpoints(a.shape, args.spacing, chip_size=chip, search_radius=radius)
    prep = ar.prepare(ar.ImagePair(a, b, None, v), p, ctx)
    dev = torch.device("cuda", 0)
    n = len(grid)
    cols = {f: torch.from_numpy(grid.flat(f)).to(dev) for f in ar.points.FIELDS}
    pts = L.ArPoints(*(cols[f].data_ptr() for f in ar.points.FIELDS), n)
    outs = [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3)]
    srch = torch.empty(n, dtype=torch.uint8, device=dev)
    h = prep.device(ctx).handle
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    def call():
        ctx.check(ctx.lib.ar_track_device(ctx.handle, h, ctypes.byref(pts), UP, L.AR_ZNCC,
                                          outs[0].data_ptr(), outs[1].data_ptr(),
                                          outs[2].data_ptr(), srch.data_ptr(), None))
    timed_steps(torch, call, stream, flush, 0, args.warmup)
    ctx.set_timing(True)
    ctx.kernel_times()
    t = timed_steps(torch, call, stream, flush, args.steps, 0)
    corr_ms, refine_ms, _, _, flops = ctx.kernel_times()
    print(json.dumps({"profile_pass": "split_bf16" if precision else "u8_fine", "points": n,
                      "kernel": args.kernel,
                      "chip": chip, "radius": radius, "ms_per_pass": t / args.steps,
                      "k_corr_ms": corr_ms / args.steps, "k_refine_ms": refine_ms / args.steps,
                      "algorithmic_tflops": flops / (corr_ms * 1e-3) / 1e12 if corr_ms else None}))


def serve_arm(args):
    """The serving configuration: a seeded Poisson stream of UInt16 pairs of sides 512, 2048,
    4096 and 10980 in proportion 8:4:2:1, each with its own grid spacing, chip and radius;
    sustained points/s of the request loop against the plain one-pair-at-a-time path, and
    p50/p99 pair latency."""
    import __graft_entry__ as ge

    ge.build()
    ar = ge.load_package()
    sc, reqs = serving_requests(ar, np.random.default_rng(7), args.steps * 15,
                                (512, 2048, N_SCALE, N), (8, 4, 2, 1))
    res = serving_measure(ar, sc, reqs, 0)
    print(json.dumps({"metric": "serving: sustained points/s and p50/p99 pair latency",
                      "value": res["batched_points_per_s"], "unit": UNIT, "n_gpus": 1,
                      "higher_is_better": True, "data": "synthetic", "serving": res}))


def reference_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import __graft_entry__ as ge

    ar = ge.load_package()
    from oracle import oracle as O

    O.build()
    a, b, valid = scene(ar, args.size)
    p = pipeline_params(ar)
    ca, cb, cv = crop(a, CROP), crop(b, CROP), crop(valid, CROP)
    rates = []
    pts = 0
    for it in range(args.warmup + args.steps):
        pts, dt, _, _ = host_pipeline(O, ar, ca, cb, cv, p)
        if it >= args.warmup:
            rates.append(pts / dt)
    value = float(np.mean(rates))
    grid = ar.build_grid(a.shape, p)
    n = len(grid)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": pts / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic",
        "config": {"workload": workload(args.size, *grid.shape), "points": n, "chip": CHIP,
                   "radius": RADIUS, "upsampling": UP, "image": [args.size, args.size],
                   "element_type": "uint16 -> uint8",
                   "same_config": False,
                   "why_a_crop": f"the whole {args.size}^2 scene ({n} grid points) takes about "
                                 f"{n / value:.0f} s per step on these cores, so each step is "
                                 f"the same pipeline on a centred {CROP}^2 crop of it"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
                         "sample": f"the same pipeline on a centred {CROP}^2 crop ({pts} grid "
                                   "points) per step (Julia is not installed; the C++ "
                                   "restatement of the reference's algorithm)",
                         "numerator": "FP64 direct sum; the reference uses single-precision "
                                      "FFTW (not installed here)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-rotation", action="store_true",
                    help="skip the rotation-search measurement")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the mixed-stream serving measurement")
    ap.add_argument("--serve", action="store_true",
                    help="only the serving measurement, on a longer stream with 10980^2 pairs")
    ap.add_argument("--size", type=int, default=N,
                    help="image side; the benchmark line uses 10980, profiles a smaller scene")
    ap.add_argument("--profile", action="store_true",
                    help="time the device steps only, autotuner off (for ncu captures); no JSON "
                         "bench line")
    ap.add_argument("--profile-precision", action="store_true",
                    help="time the chip-64 split-BF16 track pass only (for ncu captures)")
    ap.add_argument("--profile-pass", action="store_true",
                    help="time the fine chip-32 UInt8 track pass only, autotuner off "
                         "(k_corr_tc2; for ncu captures)")
    ap.add_argument("--spacing", type=int, default=SPACING,
                    help="grid spacing of a --profile run (the benchmark line always uses 8)")
    ap.add_argument("--kernel", choices=["tc2", "tc", "direct"], default=None,
                    help="UInt8 kernel of a --profile-pass run (AR_OPT_UINT8_KERNEL; default: "
                         "k_corr_tc2 where it fits)")
    ap.add_argument("--chip", type=int, default=None,
                    help="chip size of a --profile-pass run (default 32; 64 with --profile-precision)")
    ap.add_argument("--radius", type=int, default=None,
                    help="search radius of a --profile-pass run (default 25; 32 with "
                         "--profile-precision); surfaces wider than 64 run k_corr_tc")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
    elif args.profile_precision:
        profile_pass_arm(args, precision=True)
    elif args.profile_pass:
        profile_pass_arm(args, precision=False)
    elif args.serve:
        serve_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
