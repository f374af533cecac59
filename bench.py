#!/usr/bin/env python
"""Benchmark of the B200 search backend.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload NAME]

A step is one whole search (FaintTrail ft_search without candidate refinement:
background, preprocessing, the real stacking pass and its peaks, the null runs
with their rebuilt preprocessing, stacks, peaks and artefact screen, and the
tail-fit threshold) over one synthetic sequence resident in HBM. The metric is
the reference's stacking throughput, pixel x frame x motion per second
(io.cpp:316-319), here over the whole search time, not the stacking time alone.

Default workload: the full-frame plain search on one B200 -- 40 float32 frames
of 4096 x 4096, 30 s cadence, rates 0.1-2 px/min on a half-pixel grid (19,328
trial motions), 3 time-shuffled null runs (4 passes). Under torchrun each rank
runs its own sequence (a different sky field, seed 7 + rank): weak scaling, no
collective in the data path; the per-step device time is the maximum over ranks.

--workload batched-2k: a step is one search of 30 x 2048^2 frames with 64
time-shuffled null runs plus 16 injection-recovery copies of 50 objects each,
all 81 passes batched into persistent launches (ft_b200_search_batch_dev); the
same work with one pass per launch (passes_per_launch 1) is timed beside it.

--workload serving: 40 seeded search requests of uneven frame count, image size,
rate range and null runs arrive as a Poisson stream at 20 per second into the
serving loop (ft_b200_server_*); reports throughput, served searches/s and
p50 / p99 latency, beside the same requests run one after another through
ft_b200_search under the same arrival times.

The default run (N=1) adds to its one JSON line: `batched` (the batched
calibration workload, all passes batched, beside one pass per launch),
`serving` (a request stream drawn from the serving configuration, served beside
the same requests run one after another), `reference_cuda` (the reference's own
CUDA backend built for sm_100a on one pass of the full-frame frames, beside this
backend's pass of the same frames, compared bit for bit) and
`parity_vs_reference` (the device search on the crop the CPU baseline times,
compared with the reference's search() of that crop) and `stage` (the
preprocessing stage alone on 2048^2 frames at 40 and 120 frames: the static-sky
and matched-filter kernels against the HBM roofline). --no-extras skips them
(--stage-only keeps the stage part).

--workload large-sensor --once: one search of 60 x 9576 x 6388 frames with its
32 null runs (about 12 minutes), no warm-up; prints that search's time, rate,
stack-kernel rate, threshold and spans instead of the benchmark line.

--impl reference times the reference's own CPU implementation (FaintTrail
0.9.1 built from its sources, oracle/_ref) on the host's cores with all
threads, each step a bounded crop of the same workload (all frames, the full
motion grid, null runs), same metric and unit. Under torchrun only rank 0 runs it.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "pixel·frame·motion/s"
SHAPES = {0: "by frame count", 1: "32x16, 12 warps", 2: "64x8 paired columns, 12 warps", 3: "32x8, 16 warps",
          4: "32x4, 16 warps", 5: "32x16 shared maximum, 16 warps", 6: "32x16 shared maximum, 14 warps",
          7: "32x12, 16 warps", 8: "32x20 shared maximum, 16 warps"}
L2_BYTES = 126 * 1024 * 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fullframe-4k")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile-shape", type=int, default=0, help="stack kernel tile shape (0: autotuned)")
    ap.add_argument("--workers", type=int, default=2, help="serving: rounds in flight at once")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched, serving, stage and reference-CUDA parts")
    ap.add_argument("--stage-only", action="store_true", help="with --no-extras: still time the stage at 40 / 120 frames")
    ap.add_argument("--once", action="store_true",
                    help="one search of the workload without warm-up (for large-sensor with its 32 null runs); "
                         "prints its time, rate and stage spans, not the benchmark line")
    ap.add_argument("--serve-requests", type=int, default=16)
    ap.add_argument("--serve-max-adds", type=float, default=5.0e13)
    return ap.parse_args()


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms (reads only)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.lines, self.proc = gpu, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def profiled_traffic(workload):
    """DRAM bytes (read + write) per stack_batch_kernel launch for a workload, from
    the committed ncu summary (a line `traffic_bytes_per_launch[<workload>] = N`)."""
    import re
    path = os.path.join(ROOT, "profiles", "stack_batch_kernel_fullframe-1k.md")
    try:
        with open(path) as f:
            for line in f:
                mt = re.match(r"\s*traffic_bytes_per_launch\[(\S+)\]\s*=\s*([0-9.eE+]+)", line)
                if mt and mt.group(1) == workload:
                    return float(mt.group(2))
    except OSError:
        pass
    return None


def workload_desc(wl, m):
    return (f"{wl.name}: {wl.nframes} x {wl.width} x {wl.height} float32 frames, {wl.cadence_s:g} s cadence, "
            f"rates {wl.rate_px_min[0]:g}-{wl.rate_px_min[1]:g} px/min ({m} trial motions), "
            f"{wl.null_runs} null runs ({wl.null_runs + 1} passes)")


# --------------------------------------------------------------------------- reference CPU timing
def reference_search_rate(wl, frames_np, mjd, exptime, target_s=15.0, steps=1):
    """The reference CPU search (prepare + search, all host threads) on a crop of
    the workload sized to about target_s seconds. Returns adds/s, the crop side,
    the seconds of a step and the motion count."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ftoracle import Reference
    R = Reference()
    params = dict(wl.search_params())
    grid, _ = R.velocity_grid((mjd[-1] - mjd[0]) * 24.0, vmin_pxh=params["vmin_pxh"], vmax_pxh=params["vmax_pxh"],
                              grid_tol_px=params["grid_tol_px"])
    m = grid.shape[0]

    last = {}

    def run(side):
        crop = np.ascontiguousarray(frames_np[:, :side, :side])
        t0 = time.perf_counter()
        prep = R.prepare(crop, mjd, exptime, fwhm_px=params["fwhm_px"], null_runs=params["null_runs"])
        last["result"] = prep.search(backend="cpu", **params)
        last["crop"] = crop
        dt = time.perf_counter() - t0
        return m * wl.nframes * side * side * (1 + params["null_runs"]) / dt, dt
    side = 128
    rate, dt = run(side)
    # grow the crop until a step takes a few seconds, within the frame
    while dt * 4 < target_s and side * 2 <= min(wl.width, wl.height):
        side *= 2
        rate, dt = run(side)
    rates = [rate] + [run(side)[0] for _ in range(steps - 1)]
    return statistics.median(rates), side, dt, m, last


# --------------------------------------------------------------------------- parts of the default line
def crop_parity(dev, last, mjd, exptime, params, side):
    """The device search of the crop the CPU baseline timed, against the
    reference's search() result of that crop: threshold, tail fit, pooled null
    peaks, detection map and refined candidates, bit for bit."""
    ref, crop = last["result"], last["crop"]
    got = dev.search(crop, mjd, exptime, **params)
    cands = len(got["candidates"]) == len(ref["candidates"]) and all(
        np.array_equal(a, b) and fa == fb for (a, fa), (b, fb) in zip(got["candidates"], ref["candidates"]))
    checks = {"threshold": got["threshold"] == ref["threshold"] and got["method"] == ref["method"] and
              (got["null_a"], got["null_k"], got["null_inv_s2"]) == (ref["null_a"], ref["null_k"], ref["null_inv_s2"]),
              "null_peaks": bool(np.array_equal(got["null_peaks"], ref["null_peaks"])),
              "max_snr": bool(np.array_equal(got["max_snr"], ref["max_snr"], equal_nan=True)),
              "candidates": bool(cands)}
    return {"equal": all(checks.values()), "crop": f"{side}x{side} of all {crop.shape[0]} frames",
            "threshold": ref["threshold"], "null_peaks": int(len(ref["null_peaks"])),
            "candidates": int(len(ref["candidates"])), "checks": checks}


def lround(x):
    """std::lround of doubles (halves away from zero), exactly."""
    t = np.trunc(x)
    return (t + np.sign(x) * (np.abs(x - t) >= 0.5)).astype(np.int32)


def reference_cuda_measure(dev, frames, mjd, wl, grid):
    """The reference's own CUDA backend (CudaBackend::run, backend_cuda.cu:99-195,
    built for sm_100a from its sources) on one pass of the workload's frames with
    the full motion grid, beside this backend's pass of the same frames
    (ft_b200_stack_dev on the frames in HBM); both maps compared bit for bit.
    Rates are adds per second of kernel time (the reference's own timing of its
    kernel launches; CUDA events on the library stream here)."""
    import math
    import torch
    try:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from ftoracle import Reference
        R = Reference()
        if not R.cuda_available():
            return {"unavailable": "the reference CUDA backend sees no device"}
    except Exception as e:  # the reference build is test infrastructure; report, do not fail the bench
        return {"unavailable": f"reference build: {e}"}
    n, h, w = frames.shape
    mjd = np.asarray(mjd, np.float64)
    t_h = (mjd - 0.5 * (mjd[0] + mjd[-1])) * 24.0
    grid = np.ascontiguousarray(grid, np.float64)
    m = grid.shape[0]
    mc = max(3, int(math.ceil(0.7 * n)))
    dx = np.ascontiguousarray(lround(grid[:, :1] * t_h[None, :]))
    dy = np.ascontiguousarray(lround(grid[:, 1:] * t_h[None, :]))
    ms = torch.empty((h, w), dtype=torch.float32, device=frames.device)
    bv = torch.empty((h, w), dtype=torch.int32, device=frames.device)
    dev.stack_dev(frames.data_ptr(), w, h, w, n, dx, dy, mc, ms.data_ptr(), bv.data_ptr())
    dev.stack_dev(frames.data_ptr(), w, h, w, n, dx, dy, mc, ms.data_ptr(), bv.data_ptr())
    ours = dict(dev.timings()).get("kernel")
    host = frames.cpu().numpy()
    t0 = time.perf_counter()
    ref = R.stack_cuda_timed(host, t_h, grid, mc)
    wall = time.perf_counter() - t0
    equal = bool(np.array_equal(ref["max_snr"], ms.cpu().numpy(), equal_nan=True) and
                 np.array_equal(ref["best_v"], bv.cpu().numpy()))
    adds = float(m) * n * w * h
    return {"kernel": "reference stack_kernel (backend_cuda.cu:55-72, cuda_stack_core.hpp:46-80), sm_100a",
            "pass": f"{n} x {w} x {h} frames, {m} motions, min_count {mc} (one stacking pass)",
            "value": adds / ref["kernel"], "unit": METRIC + " (kernel time)",
            "seconds": {k: ref[k] for k in ("upload", "kernel", "download", "setup")}, "wall_s": wall,
            "b200_value": adds / ours if ours else None, "b200_kernel_s": ours,
            "speedup": ref["kernel"] / ours if ours else None, "bit_identical": equal}


def batched_measure(dev, local_rank):
    """The batched calibration workload: 30 x 2048^2 frames, 64 time-shuffled
    null runs and 16 injection copies of 50 objects, all 81 passes batched into
    persistent launches (ft_b200_search_batch_dev), beside the same search with
    one pass per launch (passes_per_launch 1); one warm-up, then one of each."""
    import torch
    from fainttrail_b200 import synthetic
    wl = synthetic.WORKLOADS["batched-2k"]
    frames, mjd, exptime, _ = synthetic.generate(wl, seed=7, device=f"cuda:{local_rank}")
    torch.cuda.synchronize()
    n, h, w = frames.shape
    copies = synthetic.injection_copies(wl, frames.shape, seed=11)
    params = wl.search_params()

    def run(**over):
        r, _ = dev.search_batch_dev(frames.data_ptr(), w, h, w, n, mjd, exptime, copies, maps=False,
                                    **dict(params, **over))
        return r, dict(dev.timings()), dev.launches()
    run()
    clocks = ClockSampler(local_rank)
    clocks.start()
    r, tm, nl = run()
    rp, tmp, nlp = run(passes_per_launch=1)
    clk = clocks.stop()
    m = r["n_velocities"]
    passes = 1 + wl.null_runs + len(copies)
    adds = float(m) * n * w * h * passes
    peaks, _ = measured_peaks()
    fp32_peak = dev.info()[1] * 128 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    achieved = adds / tm["kernel"] / 1e12
    same = (r["threshold"] == rp["threshold"] and np.array_equal(r["null_peaks"], rp["null_peaks"]) and
            r["peaks"] == rp["peaks"])
    del frames
    torch.cuda.empty_cache()
    return {"workload": (f"batched-2k: {n} x {w} x {h} float32 frames, {wl.cadence_s:g} s cadence, rates "
                         f"{wl.rate_px_min[0]:g}-{wl.rate_px_min[1]:g} px/min ({m} trial motions), {wl.null_runs} null "
                         f"runs + {len(copies)} injection copies x {len(copies[0])} objects ({passes} searches)"),
            "value": adds / tm["total"], "unit": METRIC, "ms_per_step": 1000.0 * tm["total"],
            "searches_per_s": passes / tm["total"], "gpu_launches": nl, "threshold_snr": r["threshold"],
            "plain": {"value": adds / tmp["total"], "ms_per_step": 1000.0 * tmp["total"],
                      "searches_per_s": passes / tmp["total"], "gpu_launches": nlp,
                      "path": "the same search, one pass per launch"},
            "speedup_vs_plain": tmp["total"] / tm["total"], "bit_identical_to_plain": bool(same),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak, "kernel": "stack_batch_kernel"},
            "clocks": clk}


def stage_measure(dev, local_rank, side=2048, counts=(40, 120), reps=3):
    """The preprocessing stage alone (ft_b200_stage_dev) on side x side frames at
    each frame count: sky-like noise with a few NaN pixels, 30 s cadence, FWHM 6
    px. Per kernel span: CUDA-event seconds (best of `reps` after a warm-up)
    and algorithmic bytes over that time against the measured HBM peak."""
    import torch
    peaks, _ = measured_peaks()
    hbm = peaks.get("hbm_gbs", 6650.0)
    out = {}
    for n in counts:
        g = torch.Generator(device=f"cuda:{local_rank}").manual_seed(5 + n)
        sub = torch.randn((n, side, side), generator=g, device=f"cuda:{local_rank}", dtype=torch.float32) * 8.0
        sub[:, ::97, ::89] = float("nan")
        filt = torch.empty_like(sub)
        t_h = (np.arange(n) - 0.5 * (n - 1)) * 30.0 / 3600.0
        best = {}
        for k in range(reps + 1):
            dev.stage_dev(sub.data_ptr(), side, side, side, n, t_h, 6.0, d_filtered=filt.data_ptr())
            if k == 0:
                continue
            for name, v in dev.timings():
                best[name] = min(best.get(name, float("inf")), v)
        torch.cuda.synchronize()
        sky_b = (8.0 * n + 4.0) * side * side
        filt_b = (8.0 * n + 8.0) * side * side
        ent = {"frames": n, "side": side, "seconds": {k: v for k, v in best.items()}}
        for key, name, b in (("sky", "static sky + residuals", sky_b), ("filter", "matched filter", filt_b)):
            if name in best:
                gbs = b / best[name] / 1e9
                ent[key] = {"achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm, "bytes_per_launch": b}
        out[f"n{n}"] = ent
        del sub, filt
        torch.cuda.empty_cache()
    return out


def once_measure(args, dev, wl, frames, mjd, exptime, params, local_rank):
    """One search (device-resident frames, all null runs) with no warm-up: the
    rate over its device time, the stack kernel's rate, the stage spans and the
    clocks. Includes the tile-shape autotuner's first probes."""
    n, h, w = frames.shape
    clocks = ClockSampler(local_rank)
    clocks.start()
    r = dev.search_dev(frames.data_ptr(), w, h, w, n, mjd, exptime, maps=False, **params)
    tm = dict(dev.timings())
    clk = clocks.stop()
    m = r["n_velocities"]
    passes = 1 + wl.null_runs
    adds = float(m) * n * w * h * passes
    print(json.dumps({"once": workload_desc(wl, m), "seconds": tm["total"], "value": adds / tm["total"],
                      "unit": METRIC, "stack_kernel": {"seconds": tm["kernel"], "adds_per_s": adds / tm["kernel"]},
                      "threshold_snr": r["threshold"], "threshold_method": r["method"],
                      "candidates": len(r["candidates"]), "spans": tm, "clocks": clk,
                      "gpu_launches": dev.launches()}), flush=True)
    dev.close()


# --------------------------------------------------------------------------- arms
def reference_arm(args):
    rank, _, world = env_rank()
    if rank != 0:
        return
    from fainttrail_b200 import synthetic
    wl = synthetic.WORKLOADS[args.workload]
    import torch
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    frames, mjd, exptime, _ = synthetic.generate(wl, seed=7, device=dev)
    side_max = min(1024, wl.width, wl.height)
    frames_np = frames[:, :side_max, :side_max].cpu().numpy()
    del frames
    t0 = time.perf_counter()
    rate, side, dt, m, _ = reference_search_rate(wl, frames_np, mjd, exptime, steps=max(1, args.steps))
    cores = os.cpu_count()
    sample = (f"reference search() (prepare + real pass + {wl.null_runs} null runs, backend cpu) on a "
              f"{side} x {side} crop of all {wl.nframes} frames, full motion grid; {dt:.1f} s per step")
    out = {"impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": 0, "ms_per_step": dt * 1000.0, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
           "config": {"workload": workload_desc(wl, m), "crop": f"{side}x{side} of every frame",
                      "parallelism": f"{cores} host threads"},
           "cpu_baseline": {"value": rate, "unit": METRIC, "cores": cores, "kind": "reference", "sample": sample},
           "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "wall_s": time.perf_counter() - t0}
    print(json.dumps(out), flush=True)


def b200_arm(args):
    import torch
    import fainttrail_b200 as ftb
    from fainttrail_b200 import synthetic
    rank, local_rank, world = env_rank()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    ftb.set_tile_shape(args.tile_shape)
    if args.workload == "serving":
        return serving_arm(args, rank, local_rank, world, dist)
    wl = synthetic.WORKLOADS[args.workload]
    params = wl.search_params()
    frames, mjd, exptime, truth = synthetic.generate(wl, seed=7 + rank, device=f"cuda:{local_rank}")
    torch.cuda.synchronize()
    n, h, w = frames.shape
    dev = ftb.Device(local_rank)
    copies = synthetic.injection_copies(wl, frames.shape, seed=11 + rank)
    batched = len(copies) > 0
    if args.once:
        return once_measure(args, dev, wl, frames, mjd, exptime, params, local_rank)

    def step(**over):
        kw = dict(params, **over)
        if batched:
            r, _ = dev.search_batch_dev(frames.data_ptr(), w, h, w, n, mjd, exptime, copies, maps=False, **kw)
        else:
            r = dev.search_dev(frames.data_ptr(), w, h, w, n, mjd, exptime, maps=False, **kw)
        return r, dict(dev.timings()), dev.launches()

    for _ in range(max(3, args.warmup)):
        r, tm, _ = step()
    m = r["n_velocities"]
    passes = 1 + wl.null_runs + len(copies)
    adds_step = float(m) * n * w * h * passes
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    totals, kernels, launches = [], [], 0
    stage = {}
    for _ in range(args.steps):
        r, tm, nl = step()
        totals.append(tm["total"])
        kernels.append(tm["kernel"])
        launches += nl
        for k, v in tm.items():
            stage[k] = stage.get(k, 0.0) + v
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    total = sum(totals)
    if dist:
        t = torch.tensor([total], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    value = world * args.steps * adds_step / total
    shape_used = args.tile_shape or ftb.tuned_shapes().get((n, m, w, h), 0)
    peaks, peak_kind = measured_peaks()
    sms = dev.info()[1]
    fp32_peak = sms * 128 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12  # non-FMA adds, TFLOP/s
    per_launch_adds = float(m) * n * w * h
    kernel_avg = sum(kernels) / (args.steps * passes)
    achieved = per_launch_adds / kernel_avg / 1e12
    hbm = peaks.get("hbm_gbs", 6650.0)
    # the HBM-bound stage kernels: algorithmic bytes per launch over their event time
    sky_bytes = (8.0 * n + 4.0) * w * h
    filt_bytes = (8.0 * n + 8.0) * w * h
    stage_roof = {}
    for name, b in (("static sky + residuals", sky_bytes), ("matched filter", filt_bytes)):
        if name in stage:
            gbs = b * passes * args.steps / stage[name] / 1e9
            stage_roof[name] = {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                                "bytes_per_launch": b}
    traffic = profiled_traffic(args.workload)

    # the same search with one pass per launch (the plain one-search-per-launch path)
    plain = None
    if batched:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, tmp, nlp = step(passes_per_launch=1)
        plain = {"ms_per_step": 1000.0 * tmp["total"], "value": adds_step / tmp["total"], "unit": METRIC,
                 "passes_per_launch": 1, "gpu_launches": nlp,
                 "searches_per_s": passes / tmp["total"], "wall_s": time.perf_counter() - t0}

    # end to end through the C ABI with host buffers: pinned frames in, maps out
    e2e = None
    if args.e2e_steps > 0:
        host = torch.empty((n, h, w), dtype=torch.float32, pin_memory=True)
        host.copy_(frames)
        host_np = host.numpy()

        def e2e_step():
            if batched:
                dev.search_batch(host_np, mjd, exptime, copies, maps=True, **params)
            else:
                dev.search(host_np, mjd, exptime, maps=True, **params)
        e2e_step()  # first call allocates
        if dist:
            dist.barrier()
        walls = []
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            e2e_step()
            walls.append(time.perf_counter() - t0)
        wall = sum(walls)
        if dist:
            t = torch.tensor([wall], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            wall = float(t.item())
        e2e = {"value": world * args.e2e_steps * adds_step / wall, "unit": METRIC,
               "h2d_bytes_per_step": 4 * n * h * w, "d2h_bytes_per_step": 8 * h * w * (1 + len(copies)),
               "ms_per_step": 1000.0 * wall / args.e2e_steps}
        del host, host_np

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            frames_np = frames[:, :1024, :1024].cpu().numpy()
            rate, side, dt, _, last = reference_search_rate(wl, frames_np, mjd, exptime)
            cpu = {"value": rate, "unit": METRIC, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"reference search() with backend cpu on a {side} x {side} crop of all {n} frames, "
                             f"full motion grid, {wl.null_runs} null runs ({dt:.1f} s)"}
            parity = crop_parity(dev, last, mjd, exptime, params, side)
        except Exception as e:  # the reference build is test infrastructure; report, do not fail the bench
            cpu = {"value": None, "unit": METRIC, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}"}
    extras = {}
    if world == 1 and not args.no_extras and not batched:
        extras["reference_cuda"] = reference_cuda_measure(dev, frames, mjd, wl, r["grid"])
        del frames
        torch.cuda.empty_cache()
        extras["batched"] = batched_measure(dev, local_rank)
        extras["serving"] = serving_measure(args, local_rank)
    if world == 1 and (args.stage_only or not args.no_extras) and not batched:
        extras["stage"] = stage_measure(dev, local_rank)
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
               "warmup": max(3, args.warmup), "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded sky/read/photon noise, log-uniform stars, movers at target S/N)",
               "config": {"workload": workload_desc(wl, m), "parallelism": f"independent searches x{world}",
                          "l2": f"inputs ({4 * n * h * w / 1e9:.1f} GB of frames) exceed the {L2_BYTES >> 20} MB L2"},
               "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                            "frac": achieved / fp32_peak, "traffic": traffic,
                            "kernel": "stack_batch_kernel (one persistent launch for all passes of a search), "
                                      "tile shape " + SHAPES.get(shape_used, str(shape_used)),
                            "peak_source": f"derived: {sms} SMs x 128 FP32 lanes x sm_max_mhz "
                                           f"{peaks.get('sm_max_mhz', 1965.0):g} MHz ({peak_kind} peaks file has no "
                                           f"FP32 figure); adds are non-FMA, one per lane per clock"},
               "stage_roofline": stage_roof,
               "stage_seconds_per_step": {k: v / args.steps for k, v in stage.items()},
               "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "gpu_launches": launches,
               "threshold_snr": r["threshold"], "threshold_method": r["method"]}
        if parity is not None:
            out["parity_vs_reference"] = parity
        out.update(extras)
        if batched:
            out["config"]["batch"] = (f"{wl.null_runs} null runs + {len(copies)} injection copies x "
                                      f"{len(copies[0])} objects (S/N {wl.snr[0]:g}-{wl.snr[1]:g}); "
                                      f"{passes} passes per step")
            out["searches_per_s"] = passes * args.steps / total
            out["plain"] = plain
            out["speedup_vs_plain"] = plain["ms_per_step"] / out["ms_per_step"]
        print(json.dumps(out), flush=True)
    dev.close()
    if dist:
        dist.destroy_process_group()


def result_digest(r):
    """threshold, peaks and a hash of both maps: equal digests = equal results"""
    import hashlib
    hs = hashlib.sha256()
    for a in (r["max_snr"], r["best_v"], r["null_peaks"]):
        hs.update(np.ascontiguousarray(a).tobytes())
    return (r["threshold"], r["method"], tuple(r["peaks"]), hs.hexdigest())


def serving_measure(args, local_rank, rank=0, world=1, dist=None):
    """The serving loop under a Poisson stream of uneven requests drawn from the
    serving configuration (synthetic.serving_requests), beside the same requests
    run one after another (first come, first served) through ft_b200_search.
    Returns the measurements as a dict."""
    import torch
    import fainttrail_b200 as ftb
    from fainttrail_b200 import synthetic
    reqs, draws = synthetic.serving_requests(count=args.serve_requests, rate_per_s=20.0, seed=2024 + rank,
                                             max_adds=args.serve_max_adds)
    inputs = []
    for k, (t_arr, wl) in enumerate(reqs):
        f, mjd, exptime, _ = synthetic.generate(wl, seed=100 + k, device=f"cuda:{local_rank}")
        inputs.append((t_arr, wl, f.cpu().numpy(), mjd, exptime))
        del f
    torch.cuda.empty_cache()
    torch.cuda.synchronize()
    dev = ftb.Device(local_rank)
    # warm-up, then the plain sequential pass: each request alone, in arrival
    # order; its latency under the same arrival times follows from the measured
    # service times (one server, first come first served)
    for t_arr, wl, f, mjd, exptime in inputs[:2]:
        dev.search(f, mjd, exptime, maps=True, **wl.search_params())
    service, alone, adds, phases = [], [], [], {}
    for t_arr, wl, f, mjd, exptime in inputs:
        t0 = time.perf_counter()
        r = dev.search(f, mjd, exptime, maps=True, **wl.search_params())
        service.append(time.perf_counter() - t0)
        for k, v in dict(dev.timings()).items():
            phases[k] = phases.get(k, 0.0) + v
        alone.append(result_digest(r))
        n, h, w = f.shape
        adds.append(float(r["n_velocities"]) * n * w * h * (1 + wl.null_runs))
    dev.close()
    finish, lat = 0.0, []
    for (t_arr, *_), sv in zip(inputs, service):
        finish = max(finish, t_arr) + sv
        lat.append(finish - t_arr)
    plain_makespan = finish  # from the stream's start, as the served run
    budget = 150.0e9
    srv = ftb.Server(local_rank, budget, max_batch=16, workers=args.workers)
    tk = [srv.submit(f, mjd, exptime, **wl.search_params()) for _, wl, f, mjd, exptime in inputs[:2]]
    for t in tk:  # warm-up round on the server's own contexts
        srv.poll(t)
    srv.close()

    def served_run():
        srv = ftb.Server(local_rank, budget, max_batch=16, workers=args.workers)
        if dist:
            dist.barrier()
        tickets = [None] * len(inputs)
        t_start = time.perf_counter()

        def submitter():
            for k, (t_arr, wl, f, mjd, exptime) in enumerate(inputs):
                d = t_arr - (time.perf_counter() - t_start)
                if d > 0:
                    time.sleep(d)
                tickets[k] = srv.submit(f, mjd, exptime, **wl.search_params())
        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        results = [result_digest(srv.poll(t, maps=True)) for t in tickets]
        t_end = time.perf_counter()
        st = srv.stats()
        srv.close()
        return t_end - t_start, st, results

    # the served stream three times (the median makespan is reported; the GPUs
    # are shared and single runs vary by about 10 %)
    clocks = ClockSampler(local_rank)
    clocks.start()
    runs = [served_run() for _ in range(3)]
    clk = clocks.stop()
    runs.sort(key=lambda r: r[0])
    makespan, st, results = runs[1]
    spread = [r[0] for r in runs]
    if dist:
        t = torch.tensor([makespan], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        makespan = float(t.item())
    total_adds = sum(adds)
    h2d = sum(4 * f.size for _, _, f, _, _ in inputs)
    d2h = sum(8 * f.shape[1] * f.shape[2] for _, _, f, _, _ in inputs)
    lat_sorted = sorted(lat)

    def pct(v, q):
        k = max(1, int(np.ceil(q * len(v))))
        return v[min(len(v), k) - 1]
    cap = args.serve_max_adds
    return {"workload": (f"serving: {len(inputs)} requests, Poisson arrivals at 20/s, frames "
                         f"{min(i[1].nframes for i in inputs)}-{max(i[1].nframes for i in inputs)}, sizes "
                         f"{min(i[1].width for i in inputs)}x{min(i[1].height for i in inputs)} to "
                         f"{max(i[1].width for i in inputs)}x{max(i[1].height for i in inputs)}, rate ranges inside "
                         f"0.1-3 px/min, 8-32 null runs, 30 s cadence, HBM budget 150 GB; drawn from the serving "
                         f"configuration with requests above {cap:.0e} pixel-frame-motion adds drawn again "
                         f"({draws - len(inputs)} of {draws} draws, {100.0 * (draws - len(inputs)) / draws:.0f} %, "
                         f"redrawn)"),
            "value": world * total_adds / makespan, "unit": METRIC, "ms_per_step": 1000.0 * makespan,
            "searches_per_s": world * len(inputs) / makespan, "p50_s": st["p50_s"], "p99_s": st["p99_s"],
            "rounds": st["rounds"], "mean_batch": st["mean_batch"], "workers": args.workers, "max_batch": 16,
            "plain": {"value": total_adds / plain_makespan, "unit": METRIC,
                      "searches_per_s": len(inputs) / plain_makespan, "p50_s": pct(lat_sorted, 0.5),
                      "p99_s": pct(lat_sorted, 0.99), "service_s_sum": sum(service), "phase_seconds": phases,
                      "path": "ft_b200_search per request, in arrival order"},
            "speedup_vs_plain": plain_makespan / makespan,
            "e2e": {"value": world * total_adds / makespan, "unit": METRIC, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "clocks": clk, "completed": st["completed"], "gpu_launches": st["launches"],
            "bit_identical_to_alone": min(sum(a == b for a, b in zip(r[2], alone)) for r in runs),
            "requests": len(inputs), "served_makespans_s": spread}


def serving_arm(args, rank, local_rank, world, dist):
    """--workload serving: the serving measurement as its own line."""
    out = serving_measure(args, local_rank, rank, world, dist)
    if rank == 0:
        line = {"metric": METRIC, "value": out["value"], "unit": METRIC, "n_gpus": world, "steps": 1, "warmup": 2,
                "ms_per_step": out["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded requests; sky/read/photon noise, stars, movers)",
                "config": {"workload": out["workload"], "parallelism": f"independent request streams x{world}",
                           "max_batch": 16, "workers": args.workers}}
        line.update({k: v for k, v in out.items() if k not in ("workload", "value", "unit", "ms_per_step")})
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        b200_arm(args)


if __name__ == "__main__":
    main()
