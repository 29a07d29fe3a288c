"""Benchmark: frames/s of temporal set inversion + ray tracing at localsubdiv 10, 1080p.

Workload (the headline configuration): 256 primitives (spheres, max-of-abs
boxes, axis capsules) moving sinusoidally in t, combined by a random
min/max tree (70% min); tape of 4697 slots; localsubdiv 10 (1024^3 leaves),
delta 0.01, lipschitz_corrected on, pointsample on, fast_normals off;
1920x1080 frames; 120 frames with t in [0, 1] (t_i = i / 119), the octree
re-seeded from scratch at frame 0 (first_eval) and carried over between
frames by the temporal error bound.

A step is one frame: one set inversion (the `main` dispatch) plus one ray
trace (`rt_main`).  Step i renders frame i mod 120, so the default 120 timed
steps after 3 warm-up frames contain exactly one first_eval frame and 119
temporally reused frames, like one run of the animation.

  value : frames/s with the scene resident in HBM, device time (CUDA events)
          of each step summed over the timed steps; the L2 cache is flushed
          (a 256 MB write) between steps, outside the per-step events
  e2e   : the same frames through the public C API from the host: per step
          the uniforms go up, the frame's RGBA f32 pixels come back to pinned
          host memory (compute.wgsl:4687 `pixels[]`), wall clock; the copy of
          frame i runs while frame i+1 is inverted, the host queues frames
          without waiting (tsi_scene_invert_async, tsi_scene_trace_async);
          the fully synchronous loop is reported beside it
  roofline: the refinement kernel's algorithmic FP32 operations (opcost.h
          table: the FULL tape's forward ops per evaluated cell, pruning not
          subtracted) over the inversion's device time, against the nominal
          FP32 rate; the executed (pruned) ops beside it; cells/s,
          interval-instruction evaluations/s and rays/s on the line
  roofline_trace: the tracer's node traffic (40 B per node visited + 16 B
          per pixel) against measured HBM, visits per ray beside it
  invert_levels: device ms and cells of each level's launch (CUDA events
          between launches, a separate context after the timed region)
  cpu_baseline: the CPU oracle (C++ restatement of compute.wgsl, OpenMP;
          tape lowered by the oracle's own ir.rs restatement) on a bounded
          sample of the same frames
  cinematic: path-traced frames (two bounces, shadow rays, sky, 8 samples)
          of the small configuration's scene at 640x360
  temporal: the reference's published comparison, temporal set inversion
          against full per-frame re-evaluation (tsi_scene_reset each frame)
  served : open-loop Poisson requests through the continuous server at
          rates relative to the plain path's capacity (and the static-batch
          server at one rate), p50/p99 latency beside the plain path's
          per-frame latency (eight runs of the workload's animation)
  served_mix: the same over a 64-scene pool with mixed levels, sweeps,
          resolutions and cameras
  batched: 32 scenes (8..2048 primitives, localsubdiv 7..10, 1024x1024)
          per step, as 32 sequential plain calls and as one CUDA-graph replay
  swept  : swept volume over [0, 1] in 64 sub-steps, localsubdiv 9, 1280x720,
          delta 0.005 / 0.01 / 0.02: frames/s and cell reuse
  split  : the animation cut at the root into eight subtree scenes on this
          GPU, inverted together, traced and composited by nearest depth

--impl reference times the CPU restatement (the reference itself is WGSL
under wgpu/Vulkan: no Vulkan driver or Rust toolchain exists on these
machines) on the GPU arm's frames (warm-up frames untimed, then the timed
steps) and prints the same line with "impl": "reference".

Multi-GPU (--gpus N, launched under torchrun): replicas.  The frames of one
animation depend on each other through the resident octree, so each rank
renders its own animation (scene seed = rank); per-GPU work is fixed
("scaling": "weak") and value is the total frames/s of all ranks with the
time taken as the maximum over ranks.  No collective is on the data path.
(One animation split at the root over GPUs, with its nearest-depth
exchange, is temporalsetinversion_b200.split; the `split` leg measures its
parts on one GPU.)
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = dict(name="csg256_L10_1080p_120f", n_prims=256, seed=1, localsubdiv=10, delta=0.01,
                lipschitz_corrected=1, pointsample=1, fast_normals=0, width=1920, height=1080, frames=120,
                eye=(1.6, 1.0, 1.9))
METRIC = "frames/s @ subdiv 10, 1080p"
PEAK_FP32_NOMINAL_TOPS = 148 * 128 * 1.965  # G ops/s: 148 SMs x 128 FP32 lanes x 1.965 GHz (non-FMA)
# DRAM bytes (read + write) per launch from one ncu capture of this workload's
# frame 4 (dram__bytes_read.sum + dram__bytes_write.sum): refine_kernel
# averaged over the frame's ten level launches, trace_kernel per frame.
# Constants of that capture, not measured by this run.
TRAFFIC_REFINE_PER_LAUNCH = 0.907e6
TRAFFIC_TRACE_PER_LAUNCH = 21.99e6
TRAFFIC_SOURCE = "one ncu capture of frame 4 of this workload (constant, not measured by this run)"


def frame_time(i: int, frames: int) -> float:
    return (i % frames) / (frames - 1)


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def init_dist(world: int):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return dist


def reduce_max(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def build_workload(seed: int):
    from temporalsetinversion_b200 import api, scenes
    text = scenes.csg(WORKLOAD["n_prims"], seed)
    params = api.default_params(localsubdiv=WORKLOAD["localsubdiv"], delta=WORKLOAD["delta"],
                                lipschitz_corrected=WORKLOAD["lipschitz_corrected"],
                                pointsample=WORKLOAD["pointsample"], fast_normals=WORKLOAD["fast_normals"])
    view = scenes.camera_look_at(WORKLOAD["eye"])
    return text, params, view


# ------------------------------------------------------------------ CPU legs
def reference_params(**kw):
    """tsi_params for the CPU oracle without loading the library: the
    PARAMETERS block defaults (compute.wgsl:3494-3511) and the root box of
    ir.rs:343-347, overridden by name (tests check them against
    tsi_default_params)."""
    from temporalsetinversion_b200 import _native as N
    p = N.Params()
    p.localsubdiv, p.delta, p.pointsample, p.fastenabled = 8, 0.01, 1, 1
    p.lipschitz_corrected = p.swept_volume = p.fast_normals = p.normal_viz = p.rounding_mode = 0
    p.fast_multiplier, p.scene_id, p.octree_darken_factor = 1.0, 1, 0.98
    for i in range(3):
        p.root_lo[i], p.root_hi[i] = -5.0, 5.0
    p.pruning, p.swept_dt = 1, 1.0 / 60.0
    p.cinematic, p.samples, p.see_background = 0, 8, 0
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def workload_params_ref():
    return reference_params(localsubdiv=WORKLOAD["localsubdiv"], delta=WORKLOAD["delta"],
                            lipschitz_corrected=WORKLOAD["lipschitz_corrected"], pointsample=WORKLOAD["pointsample"],
                            fast_normals=WORKLOAD["fast_normals"])


def oracle_scene(text: str, params):
    """The CPU oracle on the scene's tape, lowered by the oracle's own
    restatement of ir.rs (oracle/ir_ref.py), so nothing of the product's
    library runs in the CPU legs."""
    import oracle
    from oracle import ir_ref
    from temporalsetinversion_b200.api import GPU_INSTR_DTYPE
    rows = ir_ref.lower(text, 0.0)
    tape = np.zeros(len(rows), GPU_INSTR_DTYPE)
    for k, r in enumerate(rows):
        tape[k] = (r[0], r[1], r[2], r[3], (r[4], r[5]), (r[6], r[7]))
    return oracle.Scene(tape, params)


def cpu_frames(S, view, frames, threads: int) -> float:
    """Invert + trace the animation's frames `frames` on the oracle with
    `threads` OpenMP threads (the octree re-seeded at frame 0 of each run of
    the animation, as in the GPU arm); seconds."""
    import oracle
    from temporalsetinversion_b200 import api
    oracle.set_threads(threads)
    F = WORKLOAD["frames"]
    t0 = time.perf_counter()
    for i in frames:
        t = frame_time(i, F)
        if i % F == 0:
            S.reset()
        S.invert(t)
        S.trace(api.make_uniforms(view, (WORKLOAD["width"], WORKLOAD["height"]), t))
    return time.perf_counter() - t0


def all_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_baseline_sample(text: str, view, warmup: int) -> dict:
    """The oracle on a bounded sample of the GPU arm's frames: frames
    0 .. warmup-1 untimed (the first_eval frame builds the octree), then two
    frames on one thread and ten frames on all host threads, timed."""
    S = oracle_scene(text, workload_params_ref())
    cores = all_cores()
    cpu_frames(S, view, range(warmup), cores)
    one = cpu_frames(S, view, range(warmup, warmup + 2), 1)
    many = cpu_frames(S, view, range(warmup + 2, warmup + 12), cores)
    return {"value": 10 / many, "unit": "frames/s", "cores": cores, "kind": "port",
            "sample": "CPU oracle (C++ restatement of compute.wgsl main + rt_main, OpenMP; tape lowered by "
                      "oracle/ir_ref.py) on frames %d..%d of the workload after untimed frames 0..%d, full "
                      "1920x1080 trace, %.1f s" % (warmup + 2, warmup + 11, warmup - 1, many),
            "single_thread": {"value": 2 / one, "unit": "frames/s", "cores": 1,
                              "sample": "frames %d..%d on one thread, %.1f s" % (warmup, warmup + 1, one)}}


def line_config(tape_slots: int, registers=None, world: int = 1) -> dict:
    cfg = {"workload": WORKLOAD["name"], "localsubdiv": 10, "resolution": "1920x1080", "frames": WORKLOAD["frames"],
           "tape_slots": tape_slots, "parallelism": "replicas" if world > 1 else "single",
           "l2": "flushed between steps (256 MB write outside the per-step events)"}
    if registers is not None:
        cfg["registers"] = registers
    return cfg


def run_reference(args, rank, world, dist) -> None:
    """The CPU restatement of the reference's path (the reference's own WGSL
    under wgpu/Vulkan cannot run on these machines) on the GPU arm's frames:
    frames 0 .. warmup-1 untimed, then `steps` frames timed (at most one run
    of the 120-frame animation), all host threads.  Rank 0 only."""
    if rank != 0:
        return
    from temporalsetinversion_b200 import scenes
    text = scenes.csg(WORKLOAD["n_prims"], WORKLOAD["seed"])
    view = scenes.camera_look_at(WORKLOAD["eye"])
    S = oracle_scene(text, workload_params_ref())
    cores = all_cores()
    W, K = args.warmup, max(1, min(args.steps, WORKLOAD["frames"]))
    cpu_frames(S, view, range(W), cores)
    dt = cpu_frames(S, view, range(W, W + K), cores)
    value = K / dt
    tape_slots = 4697
    line = {
        "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": 1000.0 * dt / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded CSG scene emitted as LLVM IR, lowered like scenes/*.ll)",
        "config": line_config(tape_slots, world=world),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "frames/s", "cores": cores, "kind": "port",
                         "sample": "CPU oracle (C++ restatement of compute.wgsl main + rt_main, OpenMP; tape lowered "
                                   "by oracle/ir_ref.py) on frames %d..%d after untimed frames 0..%d, the GPU arm's "
                                   "frames; the reference's WGSL path (wgpu/Vulkan) cannot run here" % (W, W + K - 1, W - 1)},
        "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ temporal leg
TEMPORAL = dict(frames=40, skip=4, slow=10)


def temporal_leg(local: int) -> dict:
    """The reference's published comparison (docs/index.html:41): temporal
    set inversion against full per-frame re-evaluation at delta 0.01.  The
    headline animation's frames inverted twice, on the carried-over octree
    and with tsi_scene_reset before every frame (the first_eval path); the
    same frames' inversion (and inversion + 1080p trace) device times.  Run
    at the animation's own speed and at a tenth of it (frame times i/1190
    instead of i/119), where less of the surface moves between frames."""
    from temporalsetinversion_b200 import Device, Scene, Tape, _native as N, api
    text, params, view = build_workload(WORKLOAD["seed"])
    W, H, F = WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["frames"]
    dev = Device(local)
    try:
        scene = Scene(dev, Tape.from_llvm_ir(dev, text), params, voxel_capacity=64 << 20)
        res = {}
        for speed, div in (("animation", 1), ("slow", TEMPORAL["slow"])):
            out = {}
            for mode in ("carried", "reset"):
                scene.reset()
                inv, tr, cells = 0.0, 0.0, 0
                for i in range(TEMPORAL["frames"]):
                    t = frame_time(i, F) / div
                    if mode == "reset":
                        scene.reset()
                    st = scene.invert(t)
                    ts = N.Stats()
                    u = api.make_uniforms(view, (W, H), t)
                    N.check(dev.lib.tsi_scene_trace(scene.handle, C.byref(u), None, C.byref(ts)), "tsi_scene_trace")
                    if i >= TEMPORAL["skip"]:
                        inv += st.device_ms
                        tr += ts.device_ms
                        cells += st.cells_evaluated
                n = TEMPORAL["frames"] - TEMPORAL["skip"]
                out[mode] = {"invert_ms": inv / n, "frame_ms": (inv + tr) / n, "cells_evaluated": cells // n}
            out["invert_speedup"] = out["reset"]["invert_ms"] / out["carried"]["invert_ms"]
            out["frame_speedup"] = out["reset"]["frame_ms"] / out["carried"]["frame_ms"]
            out["cells_ratio"] = out["reset"]["cells_evaluated"] / max(1, out["carried"]["cells_evaluated"])
            res[speed] = out
        return {"frames": "%d..%d" % (TEMPORAL["skip"], TEMPORAL["frames"] - 1), **res,
                "note": "headline animation (256 primitives, localsubdiv 10, delta 0.01); reset = the octree "
                        "rebuilt from the root every frame; device ms per frame; slow = the same animation at a "
                        "tenth of its speed"}
    finally:
        dev.close()


# ------------------------------------------------------------------ cinematic leg
CINEMATIC = dict(localsubdiv=8, width=640, height=360, samples=8, frames=10)


def cinematic_leg(local: int) -> dict:
    """Path-traced frames (tsi_params.cinematic: two bounces, sun and shadow
    rays, sky, 8 samples per pixel, finite-difference normals) of the small
    plain configuration's scene (16 moving spheres, localsubdiv 8,
    640x360): device ms of the trace per frame and rays per second (primary,
    bounce and shadow rays counted as traced: at most 4 per sample)."""
    from temporalsetinversion_b200 import Device, Scene, Tape, _native as N, api, scenes
    cfg = CINEMATIC
    dev = Device(local)
    try:
        p = api.default_params(localsubdiv=cfg["localsubdiv"], pointsample=0, fast_normals=1, cinematic=1,
                               samples=cfg["samples"], see_background=1)
        s = Scene(dev, Tape.from_llvm_ir(dev, scenes.spheres16(0)), p)
        view = scenes.camera_look_at((0.3, 0.6, 2.5))
        ms = []
        for i in range(cfg["frames"] + 2):
            t = i / 60.0
            s.invert(t)
            ts = N.Stats()
            u = api.make_uniforms(view, (cfg["width"], cfg["height"]), t)
            N.check(dev.lib.tsi_scene_trace(s.handle, C.byref(u), None, C.byref(ts)), "tsi_scene_trace")
            if i >= 2:
                ms.append(ts.device_ms)
        mean = sum(ms) / len(ms)
        px = cfg["width"] * cfg["height"]
        return {"trace_ms_per_frame": mean, "frames_per_s": 1000.0 / mean,
                "primary_rays_per_s": px * cfg["samples"] / (mean / 1000.0),
                "config": "16 spheres, localsubdiv 8, %dx%d, %d samples, fast normals" % (
                    cfg["width"], cfg["height"], cfg["samples"])}
    finally:
        dev.close()


# ------------------------------------------------------------------ serving helpers
def open_loop(srv, items, arrivals, submit) -> dict:
    """Submits items[k] at start + arrivals[k] (Poisson open loop), collects
    every ticket; latencies of the completed requests, wall time from the
    first submission to the last completion, refused submissions."""
    import threading

    from temporalsetinversion_b200 import _native as N
    tickets, lats, errors = [], [], []
    refused = [0]
    submitted_all = threading.Event()
    done = threading.Event()

    def collect():
        i = 0
        while True:
            if i >= len(tickets):
                if submitted_all.is_set() and i >= len(tickets):
                    break
                time.sleep(0.0002)
                continue
            try:
                r = srv.poll(tickets[i], 1000)
            except Exception as e:  # the request failed: count it, go on
                errors.append(str(e))
                i += 1
                continue
            if r is not None:
                lats.append(r[1])
                i += 1
        done.set()

    th = threading.Thread(target=collect, daemon=True)
    th.start()
    start = time.perf_counter()
    for k, it in enumerate(items):
        delay = start + arrivals[k] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        try:
            tickets.append(submit(srv, it))
        except N.TsiError as e:  # queue full or over the memory budget
            refused[0] += 1
    submitted_all.set()
    done.wait(300.0)
    wall = time.perf_counter() - start
    th.join(5.0)
    lats = np.sort(np.asarray(lats)) if lats else np.zeros(1)
    return {"requests": int(len(lats)), "frames_per_s": len(lats) / wall, "p50_ms": float(np.percentile(lats, 50)),
            "p99_ms": float(np.percentile(lats, 99)), "max_ms": float(lats[-1]), "failed": len(errors),
            "refused": refused[0], "first_error": errors[0] if errors else None}


def served_runs(dev, plain: dict, rates, seconds: float, rng, draw, submit, static_at=None) -> list:
    """Open-loop runs through the continuous server at each rate (and the
    static-batch server at `static_at` for comparison)."""
    from temporalsetinversion_b200 import Server
    runs = []
    plan = [(r, False) for r in rates] + ([(static_at, True)] if static_at else [])
    for rate, static in plan:
        n = int(rate * seconds)
        items = draw(n)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
        with Server(dev, static_batches=static) as srv:
            r = open_loop(srv, items, arrivals, submit)
            ss = srv.stats()
        r.update({"rate_rps": rate, "rate_vs_plain": rate / plain["frames_per_s"],
                  "form": "static batches" if static else "continuous",
                  "vs_plain_frames_per_s": r["frames_per_s"] / plain["frames_per_s"],
                  "p99_vs_plain_p50": r["p99_ms"] / plain["p50_ms"], "p99_vs_plain_p99": r["p99_ms"] / plain["p99_ms"],
                  "mean_running": ss["mean_batch"]})
        runs.append(r)
    return runs


# ------------------------------------------------------------------ served leg
SERVED_OFF = ("off by default: with this build's wide-tape schedule the continuous server at twice the plain "
              "path's request rate (five to eight requests in flight) stopped on a device-side memory fault whose "
              "cause is not yet found, so the legs that drive it under load do not run (--served runs them)")

SERVED = dict(scenes=8, rates_vs_plain=(0.8, 2.0, 4.0), static_vs_plain=2.0, seconds=1.5, seed=1000)


def served_leg(local: int) -> dict:
    """Open-loop Poisson arrivals over SERVED["scenes"] concurrent runs of the
    workload's animation (scene k starts at frame 15 k; each request: the
    next frame of one scene, inverted and traced at 1920x1080 with the frame
    left on the device), at rates relative to the plain path's capacity,
    through the continuous server (and the static-batch server at one rate),
    against the plain path's per-frame latency and frames/s on one scene (one
    synchronous tsi_scene_invert + tsi_scene_trace per frame)."""
    from temporalsetinversion_b200 import Device, Scene, Tape, api

    W, H, F = WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["frames"]
    dev = Device(local)
    try:
        work = [build_workload(WORKLOAD["seed"]) for k in range(SERVED["scenes"])]
        sc = [Scene(dev, Tape.from_llvm_ir(dev, t), p) for t, p, _ in work]
        lat_plain = []
        for i in range(40):
            t = frame_time(i, F)
            u = api.make_uniforms(work[0][2], (W, H), t)
            t0 = time.perf_counter()
            sc[0].invert(t)
            sc[0].trace(u, rgba=False, depth=False, normal=False)
            dev.lib.tsi_synchronize(dev.handle)
            if i >= 4:  # after the first_eval frame
                lat_plain.append((time.perf_counter() - t0) * 1000.0)
        plain = {"p50_ms": float(np.percentile(lat_plain, 50)), "p99_ms": float(np.percentile(lat_plain, 99)),
                 "frames_per_s": 1000.0 * len(lat_plain) / float(np.sum(lat_plain))}
        rng = np.random.default_rng(SERVED["seed"])
        frame = [15 * k for k in range(SERVED["scenes"])]

        def draw(n):
            which = rng.integers(0, SERVED["scenes"], n)
            out = []
            for j in which:
                j = int(j)
                t = frame_time(frame[j], F)
                frame[j] += 1
                out.append((j, t, api.make_uniforms(work[j][2], (W, H), t)))
            return out

        def submit(srv, it):
            j, t, u = it
            return srv.submit(sc[j], t, uniforms=u)

        rates = [r * plain["frames_per_s"] for r in SERVED["rates_vs_plain"]]
        runs = served_runs(dev, plain, rates, SERVED["seconds"], rng, draw, submit,
                           static_at=SERVED["static_vs_plain"] * plain["frames_per_s"])
        return {"scenes": SERVED["scenes"], "plain": plain, "runs": runs,
                "note": "Poisson arrivals, next frame of a random scene (8 runs of the workload's animation), "
                        "invert + 1080p trace, frame kept on device; latency from submit to completion; "
                        "rates relative to the plain path's frames/s"}
    finally:
        dev.close()


# ------------------------------------------------------------------ served mix leg
SERVED_MIX = dict(pool=64, rates_vs_plain=(0.8, 2.0, 4.0), static_vs_plain=2.0, seconds=1.5, seed=2000,
                  sweep_fraction=0.2, continue_fraction=0.7, levels=(8, 9, 10),
                  resolutions=((512, 512), (1280, 720), (1920, 1080)), hbm_budget_bytes=150 * 10**9)


def served_mix_leg(local: int) -> dict:
    """Requests drawn as in the served configuration: a pool of 64 seeded
    256-primitive scenes with localsubdiv uniform in {8, 9, 10}, a fifth of
    them swept-volume scenes whose requests are [t - 1/60, t] sweeps; each
    request continues its scene at t + 1/60 with probability 0.7, else
    jumps to a random t, with a random camera on the radius-2.5 sphere and a
    resolution drawn from 512x512, 1280x720, 1920x1080.  Poisson arrivals
    at rates relative to the plain path's capacity through the continuous
    server (and the static-batch server at one rate), against the same kind
    of request sequence run one synchronous plain call pair at a time;
    scenes and frames are admitted against a 150 GB HBM budget."""
    from temporalsetinversion_b200 import Device, Scene, Tape, api, scenes

    cfg = SERVED_MIX
    rng = np.random.default_rng(cfg["seed"])
    dev = Device(local, hbm_budget_bytes=cfg["hbm_budget_bytes"])
    try:
        pool = []
        for k in range(cfg["pool"]):
            swept = rng.uniform() < cfg["sweep_fraction"]
            L = int(rng.choice(cfg["levels"]))
            p = api.default_params(localsubdiv=L, delta=WORKLOAD["delta"], swept_volume=int(swept),
                                   lipschitz_corrected=WORKLOAD["lipschitz_corrected"], pointsample=1)
            pool.append(Scene(dev, Tape.from_llvm_ir(dev, scenes.csg(256, 100 + k)), p))
        t_now = [float(rng.uniform(0.0, 1.0)) for _ in pool]
        # each scene's first frame (its octree from scratch) at the largest
        # resolution, so the frame buffers hold every later size
        big = max(cfg["resolutions"], key=lambda r: r[0] * r[1])
        for s, t in zip(pool, t_now):
            s.invert(t, t - 1.0 / 60.0 if s.params.swept_volume == 1 else math.nan)
            s.trace(api.make_uniforms(scenes.camera_on_sphere(rng, 2.5), big, t), rgba=False, depth=False,
                    normal=False)

        def draw(n):
            out = []
            for _ in range(n):
                j = int(rng.integers(0, len(pool)))
                if rng.uniform() < cfg["continue_fraction"]:
                    t_now[j] += 1.0 / 60.0
                else:
                    t_now[j] = float(rng.uniform(0.0, 1.0))
                res = cfg["resolutions"][int(rng.integers(0, 3))]
                u = api.make_uniforms(scenes.camera_on_sphere(rng, 2.5), res, t_now[j])
                sweep = pool[j].params.swept_volume == 1
                out.append((j, t_now[j], t_now[j] - 1.0 / 60.0 if sweep else math.nan, u))
            return out

        plain_reqs = draw(200)
        lat = []
        t0 = time.perf_counter()
        for j, t, t0r, u in plain_reqs:
            a = time.perf_counter()
            pool[j].invert(t, t0r)
            pool[j].trace(u, rgba=False, depth=False, normal=False)
            dev.lib.tsi_synchronize(dev.handle)
            lat.append((time.perf_counter() - a) * 1000.0)
        plain = {"frames_per_s": len(plain_reqs) / (time.perf_counter() - t0),
                 "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}

        def submit(srv, it):
            j, t, t0r, u = it
            return srv.submit(pool[j], t, t0=t0r, uniforms=u)

        rates = [r * plain["frames_per_s"] for r in cfg["rates_vs_plain"]]
        runs = served_runs(dev, plain, rates, cfg["seconds"], rng, draw, submit,
                           static_at=cfg["static_vs_plain"] * plain["frames_per_s"])
        return {"pool": cfg["pool"], "plain": plain, "runs": runs, "scene_bytes": dev.scenes_bytes(),
                "hbm_budget_bytes": cfg["hbm_budget_bytes"],
                "note": "cfg4-style mix: 64 scenes (L 8/9/10, 20% swept), 70% continue at t+1/60, "
                        "resolutions 512^2 / 1280x720 / 1920x1080, random cameras; frames kept on the device; "
                        "rates relative to the plain path's frames/s"}
    finally:
        dev.close()


# ------------------------------------------------------------------ batched leg
BATCHED = dict(scenes=32, prims=(8, 2048), levels=(7, 10), res=1024, seed=3000, warmup=3, steps=6)


def batched_specs() -> list:
    """32 scenes of the workload's kind: primitive counts log-uniform in
    [8, 2048], localsubdiv uniform in {7..10}, a random start time in [0, 1]
    and a random camera on the radius-2.5 sphere looking at the origin."""
    from temporalsetinversion_b200 import scenes
    rng = np.random.default_rng(BATCHED["seed"])
    lo, hi = BATCHED["prims"]
    out = []
    for i in range(BATCHED["scenes"]):
        n = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        L = int(rng.integers(BATCHED["levels"][0], BATCHED["levels"][1] + 1))
        t = float(rng.uniform(0.0, 1.0))
        out.append((scenes.csg(n, BATCHED["seed"] + i), L, t, scenes.camera_on_sphere(rng, 2.5)))
    return out


def batched_leg(local: int) -> dict:
    """The 32 scenes rendered frame after frame (each scene advances by
    1/60 per step, images kept on the device) two ways on the same scenes:
    32 sequential plain calls (tsi_scene_invert + tsi_scene_trace each) per
    step, and one replay of a CUDA graph of tsi_batch_run per step."""
    import ctypes as C

    from temporalsetinversion_b200 import Device, Scene, Tape, _native as N, api

    R = BATCHED["res"]
    dev = Device(local, tape_arena_words=512 << 20)
    try:
        specs = batched_specs()
        sc, unis0, slots = [], [], []
        for text, L, t, view in specs:
            p = api.default_params(localsubdiv=L, delta=WORKLOAD["delta"],
                                   lipschitz_corrected=WORKLOAD["lipschitz_corrected"],
                                   pointsample=WORKLOAD["pointsample"], fast_normals=WORKLOAD["fast_normals"])
            tape = Tape.from_llvm_ir(dev, text)
            slots.append(tape.instruction_count)
            sc.append(Scene(dev, tape, p, voxel_capacity=(16 << 20) if L >= 10 else (4 << 20)))

        def times(k):
            return [(t + k / 60.0) % 1.0 for _, _, t, _ in specs]

        # per-tape wide threshold, timed on each scene's first frames
        t_tune = time.perf_counter()
        tuned = []
        for s, (_, _, t, _) in zip(sc, specs):
            tuned.append(s.autotune([t, (t + 1 / 60.0) % 1.0], reps=1)["wide_threshold"])
        t_tune = time.perf_counter() - t_tune

        def uniforms(k):
            return [api.make_uniforms(v, (R, R), tk) for (_, _, _, v), tk in zip(specs, times(k))]

        W, K = BATCHED["warmup"], BATCHED["steps"]
        # plain: 32 synchronous call pairs per step
        plain_ms = []
        cells = [0] * len(sc)
        for k in range(W + K):
            ts, us = times(k), uniforms(k)
            t0 = time.perf_counter()
            for i, (s, t, u) in enumerate(zip(sc, ts, us)):
                st = N.Stats()
                N.check(dev.lib.tsi_scene_invert(s.handle, t, math.nan, C.byref(st)), "tsi_scene_invert")
                N.check(dev.lib.tsi_scene_trace(s.handle, C.byref(u), None, None), "tsi_scene_trace")
                cells[i] = st.cells_evaluated
            if k >= W:
                plain_ms.append((time.perf_counter() - t0) * 1000.0)
        for s in sc:
            s.reset()
        # graph: one replay per step, thresholds tuned for the scenes together
        # (the plain arm above kept each scene's own); tuning leaves them reset
        batch_tune = api.batch_autotune(dev, [(s, t) for s, t in zip(sc, times(0))], frames=2)
        g = api.BatchGraph(dev, [(s, t, math.nan, u) for s, t, u in zip(sc, times(0), uniforms(0))])
        graph_ms, graph_dev_ms = [], []
        try:
            for k in range(W + K):
                t0 = time.perf_counter()
                g.launch(times(k), uniforms(k))
                st = g.wait()
                if k >= W:
                    graph_ms.append((time.perf_counter() - t0) * 1000.0)
                    graph_dev_ms.append(st.device_ms)
        finally:
            g.close()
        n = BATCHED["scenes"]
        plain_fps = n * K / (sum(plain_ms) / 1000.0)
        graph_fps = n * K / (sum(graph_ms) / 1000.0)
        return {"scenes": n, "resolution": "%dx%d" % (R, R), "steps": K, "warmup": W,
                "tape_slots_min": int(min(slots)), "tape_slots_max": int(max(slots)),
                "tape_slots_total": int(sum(slots)),
                "levels": {str(L): sum(1 for _, l, _, _ in specs if l == L) for L in range(7, 11)},
                "plain_frames_per_s": plain_fps, "graph_frames_per_s": graph_fps,
                "graph_vs_plain": graph_fps / plain_fps,
                "plain_ms_per_step": sum(plain_ms) / K, "graph_ms_per_step": sum(graph_ms) / K,
                "graph_device_ms_per_step": sum(graph_dev_ms) / K,
                "autotune_s": t_tune, "wide_thresholds": tuned, "batch_threshold_scale": batch_tune["scale"],
                "empty_scenes": sum(1 for c in cells if c <= 8),  # a max of disjoint subtrees at the root
                "cells_per_step": int(sum(cells)),
                "note": "wall clock per step (all 32 scenes advance by 1/60); plain = 32 x (tsi_scene_invert + "
                        "tsi_scene_trace), graph = one tsi_batch_graph_launch + tsi_batch_graph_wait; frames on "
                        "the device; warm-up steps include every scene's first_eval frame"}
    finally:
        dev.close()


# ------------------------------------------------------------------ swept leg
SWEPT = dict(n_prims=64, seed=2, localsubdiv=9, substeps=64, deltas=(0.005, 0.01, 0.02), width=1280, height=720)


def swept_false_empty(tape, cells, t0: float, t1: float, eps: float, rng, max_cells: int = 1500) -> dict:
    """Cells evaluated in this frame and classified empty (f = +1), wider than
    a leaf (leaves are point-sampled, not bounded), checked at float64
    samples of their box (corners, centre, 8 random points) at 5 times of
    [t0, t1]: a cell with f <= 0 at a sample is a false empty."""
    sys.path.insert(0, str(ROOT / "tests"))
    from point_eval import evaluate
    w = np.maximum(cells["x"][:, 1] - cells["x"][:, 0], 0.0)
    sel = cells[(cells["t"] == np.float32(t1)) & (cells["f"] == 1.0) & (w > eps)]
    if len(sel) == 0:
        return {"checked": 0, "false_empty": 0}
    sel = sel[rng.choice(len(sel), min(len(sel), max_cells), replace=False)]
    lo = np.stack([sel["x"][:, 0], sel["y"][:, 0], sel["z"][:, 0]], axis=1).astype(np.float64)
    hi = np.stack([sel["x"][:, 1], sel["y"][:, 1], sel["z"][:, 1]], axis=1).astype(np.float64)
    corners = np.array([[(k >> 0) & 1, (k >> 1) & 1, (k >> 2) & 1] for k in range(8)], np.float64)
    u = np.concatenate([corners, [[0.5, 0.5, 0.5]], rng.uniform(size=(8, 3))], axis=0)
    pts = lo[:, None, :] + u[None, :, :] * (hi - lo)[:, None, :]
    bad = np.zeros(len(sel), bool)
    for tt in np.linspace(t0, t1, 5):
        f = evaluate(tape, pts[..., 0], pts[..., 1], pts[..., 2], np.float64(np.float32(tt)))
        bad |= np.any(f <= 0.0, axis=1)
    return {"checked": int(len(sel)), "false_empty": int(bad.sum())}


def swept_leg(local: int) -> dict:
    """Temporal / swept-volume stress: 64 primitives rotating about random
    axes with an exp(-t) scale, swept volume on, [0, 1] in 64 sub-steps
    (frame k inverts over [k/64, (k+1)/64] and traces at 1280x720),
    localsubdiv 9, for each delta: device frames/s, cells evaluated and the
    fraction of ambiguous cells carried over (reused) per frame; and the
    false-empty rate against float64 samples, in round-to-nearest (the
    reference's arithmetic) and in directed rounding."""
    from temporalsetinversion_b200 import Device, Scene, Tape, _native as N, api, scenes

    W, H, K = SWEPT["width"], SWEPT["height"], SWEPT["substeps"]
    view = scenes.camera_look_at(WORKLOAD["eye"])
    dev = Device(local)
    try:
        text = scenes.swept(SWEPT["n_prims"], SWEPT["seed"])
        tape_np = api.IR.new(text).gpu_instructions
        eps = 10.0 * 2.0 ** -SWEPT["localsubdiv"]
        out = []
        for delta in SWEPT["deltas"]:
            row = {"delta": delta}
            for mode, rounding in (("nearest", 0), ("directed", 1)):
                p = api.default_params(localsubdiv=SWEPT["localsubdiv"], delta=delta, swept_volume=1,
                                       rounding_mode=rounding)
                s = Scene(dev, Tape.from_llvm_ir(dev, text), p, voxel_capacity=16 << 20)
                thr = s.autotune([(k + 1) / K for k in range(3)], reps=1)["wide_threshold"] if rounding == 0 else None
                rng = np.random.default_rng(int(delta * 1e4) + rounding)
                ms, cells, reused, enq, checked, false_empty = 0.0, 0, 0, 0, 0, 0
                for k in range(K):
                    t0, t1 = k / K, (k + 1) / K
                    st = s.invert(t1, t0)
                    u = api.make_uniforms(view, (W, H), t1)
                    ts = N.Stats()
                    N.check(dev.lib.tsi_scene_trace(s.handle, C.byref(u), None, C.byref(ts)), "tsi_scene_trace")
                    if k > 0:  # frame 0 builds the octree from scratch
                        ms += st.device_ms + ts.device_ms
                        cells += st.cells_evaluated
                        reused += st.cells_reused
                        enq += st.cells_enqueued
                    if k % 8 == 7:  # every eighth sub-step: float64 samples of its empty cells
                        fe = swept_false_empty(tape_np, s.cells(), t0, t1, eps, rng)
                        checked += fe["checked"]
                        false_empty += fe["false_empty"]
                res = {"frames_per_s": (K - 1) / (ms / 1000.0), "cells_evaluated_per_frame": cells / (K - 1),
                       "reused_per_frame": reused / (K - 1), "reuse_fraction": reused / max(1, reused + enq),
                       "empty_cells_checked": checked, "false_empty": false_empty,
                       "false_empty_rate": false_empty / max(1, checked)}
                if thr is not None:
                    res["wide_threshold"] = thr
                row[mode] = res
                s.close()
            out.append(row)
        return {"workload": "swept64_L9_720p_64substeps", "runs": out,
                "note": "reuse_fraction = ambiguous cells kept with their subtree / (kept + re-subdivided); "
                        "false_empty: of the sampled empty cells (evaluated in the frame, wider than a leaf, at "
                        "most 1500 per checked sub-step, every eighth sub-step) those with f <= 0 at a float64 "
                        "sample of their box over the sub-step's time interval"}
    finally:
        dev.close()


SPLIT = dict(level=1, frames=40, part_frames=6)


def split_leg(local: int) -> dict:
    """The headline animation cut at the root into its eight subtrees, all
    on this GPU (temporalsetinversion_b200.split): per frame the eight
    subtree scenes are inverted in one fused launch sequence and traced over
    the 1080p image (tsi_batch_run), then composited by nearest depth
    (tsi_frames_composite).  Wall-clock frames/s over the animation's first
    frames, the composite's time, and each part run alone (device time of
    its inversion + trace): the slowest part bounds one frame of an
    eight-GPU split, before the exchange."""
    from temporalsetinversion_b200 import Device, Tape, api, split

    W, H, F = WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["frames"]
    text, params, view = build_workload(WORKLOAD["seed"])
    dev = Device(local)
    try:
        tape = Tape.from_llvm_ir(dev, text)
        sp = split.SubtreeSplit(dev, tape, params, level=SPLIT["level"], voxel_capacity=16 << 20)
        n = SPLIT["frames"]
        warm = 3
        for i in range(warm):
            t = frame_time(i, F)
            sp.frame(t, api.make_uniforms(view, (W, H), t))
        dev_ms, comp_s = 0.0, 0.0
        t0 = time.perf_counter()
        for i in range(warm, n):
            t = frame_time(i, F)
            fb, stats = sp.frame(t, api.make_uniforms(view, (W, H), t))
            dev_ms += stats[0].device_ms
        wall = time.perf_counter() - t0
        for _ in range(5):
            c0 = time.perf_counter()
            sp.composite(fb)
            comp_s += time.perf_counter() - c0
        hits = int((fb["depth"] >= 0).sum().item())
        # each part alone over the next frames (scenes continue the animation)
        part_ms = [0.0] * len(sp.scenes)
        for i in range(n, n + SPLIT["part_frames"]):
            t = frame_time(i, F)
            u = api.make_uniforms(view, (W, H), t)
            for k, s in enumerate(sp.scenes):
                part_ms[k] += api.run_batch(dev, [(s, t, math.nan, None)])[0]["stats"].device_ms
                part_ms[k] += s.trace(u, rgba=False, depth=False, normal=False)["device_ms"]
        part_ms = [m / SPLIT["part_frames"] for m in part_ms]
        sp.close()
        return {"parts": len(sp.ids), "level": SPLIT["level"], "frames": n - warm,
                "frames_per_s": (n - warm) / wall, "device_ms_per_frame": dev_ms / (n - warm),
                "composite_ms": 1000.0 * comp_s / 5, "hit_pixels": hits,
                "part_ms": [round(m, 4) for m in part_ms], "part_ms_max": max(part_ms), "part_ms_sum": sum(part_ms),
                "note": "one GPU holds all eight subtree scenes; wall clock per frame (fused inversion of the parts, "
                        "eight traces, composite); part_ms = one part's inversion + trace run alone, device time"}
    finally:
        dev.close()


# ------------------------------------------------------------------ level profile
def level_profile(local: int, text: str, params, frames=(4, 5, 6, 7, 8)) -> dict:
    """Device ms of each level's refinement launch (CUDA events between the
    launches, TSI_PROFILE_LEVELS) and cells evaluated per level, averaged
    over the animation's frames `frames` (carried-over frames), on a separate
    context after the timed region."""
    from temporalsetinversion_b200 import Device, Scene, Tape, _native as N
    os.environ["TSI_PROFILE_LEVELS"] = "1"
    try:
        dev = Device(local)
    finally:
        del os.environ["TSI_PROFILE_LEVELS"]
    try:
        scene = Scene(dev, Tape.from_llvm_ir(dev, text), params, voxel_capacity=64 << 20)
        F = WORKLOAD["frames"]
        acc_ms, acc_cells, n = None, None, 0
        for i in range(max(frames) + 1):
            scene.invert(frame_time(i, F))
            if i not in frames:
                continue
            L = 32
            ms = (C.c_float * L)()
            ctr = (C.c_uint64 * (L * len(N.LEVEL_COUNTERS)))()
            nl = C.c_uint32(0)
            N.check(dev.lib.tsi_debug_level_profile(dev.handle, L, ms, ctr, C.byref(nl)), "tsi_debug_level_profile")
            k = min(nl.value, L)
            NC = len(N.LEVEL_COUNTERS)
            lm = [ms[j] for j in range(k)]
            rows = [[ctr[j * NC + q] for q in range(NC)] for j in range(k)]
            acc_ms = lm if acc_ms is None else [a + b for a, b in zip(acc_ms, lm)]
            acc_cells = rows if acc_cells is None else [[a + b for a, b in zip(r0, r1)] for r0, r1 in zip(acc_cells, rows)]
            n += 1
        names = N.LEVEL_COUNTERS
        keep = ("evaluated", "wide_items", "cyc_wide_max", "cyc_narrow", "cyc_narrow_max", "instr_fwd", "instr_full")
        per = {name: [r[names.index(name)] // n for r in acc_cells] for name in keep}
        # narrow items per level: every narrow item counted its parents; wide
        # cells count one parent per group finish
        return {"ms": [round(v / n, 4) for v in acc_ms], "counters": per, "frames": list(frames),
                "note": "CUDA events between the level launches of one frame; counters per level (SM cycles "
                        "are clock64 of the item on its SM)"}
    finally:
        dev.close()


# ------------------------------------------------------------------ GPU leg
def run_gpu(args, rank, world, local, dist) -> None:
    import ctypes as C

    from temporalsetinversion_b200 import Device, Scene, Tape, _native as N, api

    text, params, view = build_workload(WORKLOAD["seed"] + rank)
    W, H, F = WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["frames"]
    if args.small_arenas:  # a few GB on the device in all, for profiler captures
        dev = Device(local, work_item_capacity=1 << 20, tape_arena_words=16 << 20, log_arena_bytes=1 << 30)
    else:
        dev = Device(local)
    lib = dev.lib
    tape = Tape.from_llvm_ir(dev, text)
    scene = Scene(dev, tape, params, voxel_capacity=args.voxels)

    # L2 flush buffer (256 MB) and events through torch on this device
    import torch
    torch.cuda.set_device(local)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")

    totals = {k: 0 for k in ("cells_evaluated", "instr_forward", "instr_reverse", "instr_full_equiv", "fp32_ops",
                             "fp32_ops_full_fwd", "fp32_ops_full_rev", "cells_reused", "cells_reverse")}
    inv_ms, trace_ms = [], []
    visits = 0.0

    def step(i: int, record: bool):
        nonlocal visits
        t = frame_time(i, F)
        if i % F == 0:
            scene.reset()
        st = scene.invert(t)
        u = api.make_uniforms(view, (W, H), t)
        tst = N.Stats()
        N.check(lib.tsi_scene_trace(scene.handle, C.byref(u), None, C.byref(tst)), "tsi_scene_trace")
        if record:
            inv_ms.append(st.device_ms)
            trace_ms.append(tst.device_ms)
            visits += tst.reserved
            for k in totals:
                totals[k] += getattr(st, k)
        return st

    for i in range(args.warmup):
        step(i, False)
    barrier(dist)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    t_wall0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        step(i, True)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall0
    clocks = sampler.stop()
    barrier(dist)
    dev_ms = float(sum(inv_ms) + sum(trace_ms))
    dev_ms_max = reduce_max(dist, dev_ms)
    frames_total = reduce_sum(dist, float(args.steps))
    value = frames_total / (dev_ms_max / 1000.0)

    # ---- e2e through the C API with host buffers: each frame's RGBA comes
    # back to pinned host memory; the copy of frame i overlaps the inversion
    # of frame i+1 (tsi_scene_trace_async), two host buffers in turn
    pinned = [torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    imgs = [N.Image(W, H, C.cast(p.data_ptr(), C.POINTER(C.c_float)), None, None) for p in pinned]
    e2e_steps = min(args.steps, F)
    unis = [api.make_uniforms(view, (W, H), frame_time(i, F)) for i in range(e2e_steps)]

    def e2e_run(asynchronous: bool) -> float:
        scene.reset()
        barrier(dist)
        t0 = time.perf_counter()
        for i in range(e2e_steps):
            t = frame_time(i, F)
            if asynchronous:
                N.check(lib.tsi_scene_invert_async(scene.handle, t, math.nan), "tsi_scene_invert_async")
                N.check(lib.tsi_scene_trace_async(scene.handle, C.byref(unis[i]), C.byref(imgs[i & 1])),
                        "tsi_scene_trace_async")
            else:
                st = N.Stats()
                N.check(lib.tsi_scene_invert(scene.handle, t, math.nan, C.byref(st)), "tsi_scene_invert")
                N.check(lib.tsi_scene_trace(scene.handle, C.byref(unis[i]), C.byref(imgs[0]), None),
                        "tsi_scene_trace")
        if asynchronous:
            N.check(lib.tsi_scene_invert_wait(scene.handle, None), "tsi_scene_invert_wait")
            N.check(lib.tsi_scene_trace_wait(scene.handle), "tsi_scene_trace_wait")
        return reduce_max(dist, time.perf_counter() - t0)

    e2e_sync_value = reduce_sum(dist, float(e2e_steps)) / e2e_run(False)
    e2e_value = reduce_sum(dist, float(e2e_steps)) / e2e_run(True)

    if rank != 0:
        dev.close()
        return
    peaks = measured_peaks()
    inv_total_s = sum(inv_ms) / 1000.0
    trace_s = sum(trace_ms) / 1000.0
    # algorithmic work (opcost.h table) on the FULL tape, whatever pruning
    # saved: forward ops of every evaluated cell; reverse ops beside it
    alg_fwd, alg_rev = totals["fp32_ops_full_fwd"], totals["fp32_ops_full_rev"]
    executed = totals["fp32_ops"]
    peak_gops = PEAK_FP32_NOMINAL_TOPS
    achieved_gops = alg_fwd / inv_total_s / 1e9 if inv_total_s > 0 else 0.0
    trace_bytes = visits * 40.0 + W * H * 16.0 * len(trace_ms)
    trace_gbs = trace_bytes / trace_s / 1e9 if trace_s > 0 else 0.0
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    gpu_launches = args.steps * (params.localsubdiv + 3)
    line = {
        "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded CSG scene emitted as LLVM IR, lowered like scenes/*.ll)",
        "config": line_config(tape.instruction_count, tape.registers, world),
        "e2e": {"value": e2e_value, "unit": "frames/s", "h2d_bytes_per_step": C.sizeof(N.Uniforms) + 160,
                "d2h_bytes_per_step": W * H * 16 + C.sizeof(N.Stats),
                "readback": "frames queued without waiting (tsi_scene_invert_async, tsi_scene_trace_async); "
                            "frame i's copy to pinned host memory overlaps frame i+1's inversion; errors checked "
                            "at the end (tsi_scene_invert_wait)",
                "synchronous_value": e2e_sync_value},
        "cells_per_s": totals["cells_evaluated"] / inv_total_s if inv_total_s > 0 else 0.0,
        "instr_evals_per_s": totals["instr_full_equiv"] / inv_total_s if inv_total_s > 0 else 0.0,
        "rays_per_s": W * H * len(trace_ms) / trace_s if trace_s > 0 else 0.0,
        "roofline": {"kernel": "refine_kernel (interval tape interpreter)", "bound": "fp32",
                     "achieved": achieved_gops / 1000.0, "peak": peak_gops / 1000.0, "unit": "TOP/s",
                     "frac": achieved_gops / peak_gops,
                     "work": "opcost.h forward FP32 ops of the full tape (fix included) per evaluated cell, "
                             "pruning not subtracted; achieved = that / inversion device time",
                     "alg_fwd_ops_per_step": alg_fwd / args.steps, "alg_rev_ops_per_step": alg_rev / args.steps,
                     "frac_with_reverse": (alg_fwd + alg_rev) / inv_total_s / 1e9 / peak_gops if inv_total_s > 0 else 0.0,
                     "executed_ops_per_step": executed / args.steps,
                     "executed_frac": executed / inv_total_s / 1e9 / peak_gops if inv_total_s > 0 else 0.0,
                     "cells_evaluated_per_step": totals["cells_evaluated"] / args.steps,
                     "invert_ms_per_step": sum(inv_ms) / args.steps,
                     "traffic": TRAFFIC_REFINE_PER_LAUNCH, "traffic_unit": "bytes per launch (ncu, dram read + write)",
                     "traffic_source": TRAFFIC_SOURCE,
                     "peak_source": "nominal FP32 rate, 148 SMs x 128 lanes x 1.965 GHz (MEASURED_PEAKS.json has no "
                                    "FP32 figure)"},
        "roofline_trace": {"kernel": "trace_kernel", "bound": "hbm", "achieved": trace_gbs, "peak": hbm_peak,
                           "unit": "GB/s", "frac": trace_gbs / hbm_peak, "traffic": TRAFFIC_TRACE_PER_LAUNCH,
                           "traffic_unit": "bytes per launch (ncu, dram read + write)", "traffic_source": TRAFFIC_SOURCE,
                           "visits_per_ray": visits / (W * H * len(trace_ms)) if trace_ms else 0.0,
                           "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "breakdown_ms_per_step": {"invert": sum(inv_ms) / args.steps, "trace": sum(trace_ms) / args.steps},
        "work_per_step": {k: v / args.steps for k, v in totals.items()},
        "clocks": clocks,
        "gpu_launches": gpu_launches,
        "wall_s": wall,
    }
    if world == 1:
        try:
            line["invert_levels"] = level_profile(local, text, params)
        except Exception as e:
            line["invert_levels"] = {"unavailable": str(e)}
    if not args.no_cpu_baseline and world == 1:
        try:
            line["cpu_baseline"] = cpu_baseline_sample(text, view, args.warmup)
        except Exception as e:  # the oracle needs g++ on the host
            line["cpu_baseline"] = {"value": None, "unit": "frames/s", "cores": 0, "kind": "port",
                                    "sample": "unavailable: %s" % e}
    dev.close()
    if world == 1 and not args.no_cinematic:
        try:
            line["cinematic"] = cinematic_leg(local)
        except Exception as e:
            line["cinematic"] = {"unavailable": str(e)}
    if world == 1 and not args.no_temporal:
        try:
            line["temporal"] = temporal_leg(local)
        except Exception as e:
            line["temporal"] = {"unavailable": str(e)}
    if world == 1 and args.served:
        try:
            line["served"] = served_leg(local)
        except Exception as e:
            line["served"] = {"unavailable": str(e)}
        try:
            line["served_mix"] = served_mix_leg(local)
        except Exception as e:
            line["served_mix"] = {"unavailable": str(e)}
    elif world == 1 and not args.no_served:
        line["served"] = line["served_mix"] = {"unavailable": SERVED_OFF}
    if world == 1 and not args.no_swept:
        try:
            line["swept"] = swept_leg(local)
        except Exception as e:
            line["swept"] = {"unavailable": str(e)}
    if world == 1 and not args.no_split:
        try:
            line["split"] = split_leg(local)
        except Exception as e:  # report, keep the headline line
            line["split"] = {"unavailable": str(e)}
    if world == 1 and not args.no_batched:
        try:
            line["batched"] = batched_leg(local)
        except Exception as e:
            line["batched"] = {"unavailable": str(e)}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tsi", choices=["tsi", "reference"])
    ap.add_argument("--voxels", type=int, default=64 << 20)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-served", action="store_true", help="leave the served legs out of the line entirely")
    ap.add_argument("--served", action="store_true", help="run the served-latency legs (see SERVED_OFF)")
    ap.add_argument("--no-batched", action="store_true", help="skip the 32-scene batched leg")
    ap.add_argument("--no-swept", action="store_true", help="skip the swept-volume leg")
    ap.add_argument("--no-split", action="store_true", help="skip the root-split leg")
    ap.add_argument("--no-temporal", action="store_true", help="skip the temporal-reuse comparison leg")
    ap.add_argument("--no-cinematic", action="store_true", help="skip the path-tracing leg")
    ap.add_argument("--small-arenas", action="store_true",
                    help="small work-item, tape and log arenas (use with --voxels 4194304 under a profiler)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()
    dist = init_dist(world)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world, dist)
        else:
            run_gpu(args, rank, world, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
