#!/usr/bin/env python
"""Benchmark: points/s of the dense ZNCC track pass on B200.

Workload (one step): the fine track pass of AutoRIFT.jl (`track`, src/track.jl:103-152) at
chip 32, search radius 25, PyramidRefine(64), ZNCC, over the 490 x 490 grid (spacing 8,
margin from chip_size_max 128) of a 4096^2 synthetic 8-bit pair (filtered noise, mean 128,
std 40; secondary warped by a 6-bump field up to 15 px, 2% noise, 3% no-data blobs masked
invalid). The two 16.8 MB images fit in L2, so L2 is flushed before every timed step by writing
a 256 MiB buffer (outside the timed interval).

Arms:
  default            our library (libautorift_gpu.so, sm_100a), N GPUs as N independent
                     replicas (one pair per rank, no collective on the data path).
  --impl reference   the reference's algorithm on the host cores: Julia is not installed, so
                     the CPU restatement (oracle/, C++ + OpenMP, all host threads) times a
                     bounded sample of the same workload.

Prints one JSON line (rank 0).
"""

from __future__ import annotations

import argparse
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
CHIP, RADIUS, UP, SPACING, N = 32, 25, 64, 8, 4096
WORKLOAD = (f"track pass (fine, ZNCC, chip {CHIP}, radius {RADIUS}, PyramidRefine({UP})) over the "
            f"490x490 spacing-{SPACING} grid of a {N}^2 synthetic UInt8 pair")


def load_workload(ar, spacing=SPACING):
    a, b, valid, _ = ar.synthetic.scale_u16_pair(N, mean=128.0, std=40.0, dtype=np.uint8)
    pts = ar.gridpoints((N, N), spacing, chip_size=4 * CHIP, search_radius=RADIUS)
    pts = ar.pointset(pts.x, pts.y, chip_size=CHIP, search_radius=RADIUS)
    return a, b, valid, pts


def flops_per_point():
    # Algorithmic FLOPs of one point evaluation: 2 * chip area * surface size.
    return 2.0 * CHIP * CHIP * (2 * RADIUS) * (2 * RADIUS)


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


def profile_traffic():
    """DRAM bytes per launch of the correlation kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "k_corr_traffic.json"
    try:
        d = json.loads(f.read_text())
        return d.get("bytes_per_point") * d.get("points_per_launch_full", 0) or None
    except (OSError, ValueError, TypeError):
        return None


def oracle_rate(O, a, b, valid, pts, target_s=12.0):
    """Points/s of the oracle (all host threads) over a random sample sized for ~target_s."""
    from autorift_b200.points import FIELDS

    n = len(pts)
    rng = np.random.default_rng(0)
    order = rng.permutation(n)

    def run(k):
        idx = order[:k]
        sub = {f: pts.flat(f)[idx] for f in FIELDS}
        t = time.perf_counter()
        O.track(a, b, sub, upsampling=UP, secondary_valid=valid, nthreads=0)
        return time.perf_counter() - t

    k = 64
    dt = run(k)
    while dt < 1.0 and k < n:
        k = min(n, k * 4)
        dt = run(k)
    k2 = int(min(n, max(k, k * target_s / max(dt, 1e-6))))
    if k2 > k:
        k, dt = k2, run(k2)
    return k / dt, k, dt


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
    ctx = ar._lib.Context(local)
    a, b, valid, pts = load_workload(ar, args.spacing)
    n = len(pts)
    pair = ar.ImagePair(a, b, None, valid)
    dp = pair.device(ctx)
    dev = torch.device("cuda", local)
    cols = {f: torch.from_numpy(pts.flat(f)).to(dev) for f in ar.points.FIELDS}
    dpts = ar._lib.ArPoints(*(cols[f].data_ptr() for f in ar.points.FIELDS), n)
    out = [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(3)]
    searched = torch.empty(n, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # A created stream: its handle is non-null, so the library launches on it (a null handle
    # would mean the library's own stream) and the events below bracket exactly its kernels.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    import ctypes

    def step():
        ctx.check(ctx.lib.ar_track_device(
            ctx.handle, dp.handle, ctypes.byref(dpts), UP, ar._lib.AR_ZNCC,
            out[0].data_ptr(), out[1].data_ptr(), out[2].data_ptr(), searched.data_ptr(),
            ctypes.c_void_p(stream.cuda_stream)))

    for _ in range(args.warmup):
        flush.fill_(1)
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ctx.set_timing(True)
    ctx.kernel_times()
    total_ms = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)  # L2 flush outside the timed interval of each step
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            step()
            e.record(stream)
            e.synchronize()
            total_ms += s.elapsed_time(e)
    torch.cuda.synchronize()
    corr_ms, refine_ms, tracks, launches, corr_flops = ctx.kernel_times()
    ctx.set_timing(False)
    t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if dist:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * n * args.steps / (total_ms * 1e-3)

    nsearched = int(searched.sum().item())
    fin = torch.isfinite(out[0])
    med_dx = float(out[0][fin].median().item()) if fin.any() else float("nan")

    # Roofline of the dominant kernel (the correlation): algorithmic FLOPs per launch (counted
    # by the kernel: 2 * chip area * surface area per searched point) over its event-timed
    # average duration, against the measured cuBLAS FP32 rate.
    corr_avg = corr_ms / max(tracks, 1)
    flops_launch = corr_flops / max(tracks, 1)
    assert abs(flops_launch - flops_per_point() * nsearched) <= 1e-9 * flops_launch + 1, \
        (flops_launch, flops_per_point() * nsearched)
    achieved = flops_launch / (corr_avg * 1e-3) / 1e12
    if args.profile:  # an ncu capture: the device steps only
        if rank == 0:
            print(json.dumps({"profile_run": True, "points": n, "ms_per_step": ms_per_step,
                              "k_corr_ms": corr_avg, "k_refine_ms": refine_ms / max(tracks, 1)}))
        if dist:
            dist.destroy_process_group()
        return
    fp32_peak = measure_fp32_peak(torch, dev)
    traffic = profile_traffic()

    # End to end through the C ABI with host buffers (pair upload, point upload, download).
    host_pts = pts
    e2e_times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        p2 = ar.ImagePair(a, b, None, valid)
        d = ar.track(p2, host_pts, ar.params(preprocess="none", quantize="none", upsampling=UP),
                     ctx=ctx)
        p2._device.clear()
        t1 = time.perf_counter()
        if it >= args.warmup:
            e2e_times.append(t1 - t0)
    e2e_value = world * n / float(np.mean(e2e_times))
    e2e_p50 = float(np.percentile(e2e_times, 50)) * 1e3
    e2e_p99 = float(np.percentile(e2e_times, 99)) * 1e3
    h2d = a.nbytes + b.nbytes + 2 * a.size + n * 48
    d2h = n * 13

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        rate, k, dt = oracle_rate(O, a, b, valid, pts)
        cpu = {"value": rate, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
               "sample": f"{k} of {n} points of the same workload, {dt:.1f} s"}

    peaks = measured_peaks()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "points": n, "searched": nsearched,
                       "chip": CHIP, "radius": RADIUS, "upsampling": UP, "image": [N, N],
                       "element_type": "uint8", "l2": "flushed (256 MiB write) between steps",
                       "parallelism": f"{world} independent replicas",
                       "median_dx": med_dx},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                         "unit": "TFLOP/s", "frac": achieved / fp32_peak if fp32_peak else None,
                         "traffic": traffic, "kernel": "k_corr",
                         "peak_source": "measured cuBLAS FP32 SGEMM (TF32 off) in this run; "
                                        "no FP32 figure in MEASURED_PEAKS.json",
                         "kernel_ms": {"k_corr": corr_avg, "k_refine": refine_ms / max(tracks, 1)},
                         "measured_peaks": {k: peaks.get(k) for k in ("hbm_gbs", "bf16_tflops")}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "p50_ms": e2e_p50, "p99_ms": e2e_p99,
                    "path": "ar_pair_upload + ar_track (host buffers) per step"},
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def reference_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import __graft_entry__ as ge

    ar = ge.load_package()
    from oracle import oracle as O

    O.build()
    a, b, valid, pts = load_workload(ar)
    n = len(pts)
    rates = []
    for it in range(args.warmup + args.steps):
        rate, k, dt = oracle_rate(O, a, b, valid, pts, target_s=max(2.0, 30.0 / (args.steps + args.warmup)))
        if it >= args.warmup:
            rates.append(rate)
    value = float(np.mean(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": n / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "points": n, "chip": CHIP, "radius": RADIUS,
                   "upsampling": UP, "image": [N, N], "element_type": "uint8"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.max_threads(), "kind": "port",
                         "sample": f"{k} of {n} points per step (Julia is not installed; the "
                                   "C++ restatement of the reference's algorithm)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--spacing", type=int, default=SPACING,
                    help="grid spacing; the benchmark line uses 8, profiles use a sparser grid")
    ap.add_argument("--profile", action="store_true",
                    help="time the device steps only (for ncu captures); no JSON bench line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
