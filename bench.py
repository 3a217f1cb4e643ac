"""Benchmark of the wavefront path-tracing loop (one JSON line on rank 0).

Headline workload (N=1): the instanced PBR scene — 64 instances of a
16,384-triangle sphere, a 2-triangle ground and 1,024 emissive triangles
(1,049,602 triangles) — at 1920x1080, 4 spp, 8 bounces, ReSTIR DI with 32
candidates, 1 temporal and 1 spatial pass (5 neighbours, radius 30 px).  A
step renders one frame.  Metric: Mrays/s (camera + extension + shadow rays
per second).

* ``value``: device time of the frame (CUDA events on the renderer's stream),
  scene resident, output into a device buffer; L2 flushed between steps.
* ``e2e``: the same frames through ``render_frame`` (host output array,
  per-step device->host image copy), timed by the host clock.
* ``roofline``: the dominant kernel's algorithmic bytes per launch over its
  average event-timed launch duration, against MEASURED_PEAKS.json.
* ``cpu_baseline``: the oracle restatement of CpuReferenceRenderer on all
  host cores, rendering config 2 scaled for its brute-force intersector
  (4 x 1,280-tri spheres, 5,138 tris) in full: camera rays and every
  extension segment of 8 bounces, nothing extrapolated; ``scaled_c2`` is the
  CUDA renderer on that scene with the same transport.
* ``served``: the served form on Poisson request streams of 5-200 req/s over
  8 resident scenes of 10k-8M triangles (p50/p99 latency, throughput,
  rejections), beside the plain path serving the same streams one request at
  a time; ``served`` is the 200 req/s point, ``served_sweep`` all of them.
* ``targets``: the north star's ratios (config 1 over the CPU reference,
  batched and served over the plain per-request path).
* ``batched``: 64 jobs over nine rescaled configuration scenes in one
  wavefront after the launch-shape autotuner, beside the same jobs one at a
  time.
* ``config1`` / ``config3``: the closed-box room against the CPU reference
  (reference-compatible mode, closest-hit rays) and the terrain with its
  delta-tracked volume.

``--impl reference`` times that CPU reference alone (rank 0): each step one
full render of the scaled config-2 scene per host core.
For N > 1 (torchrun), every rank renders its own frames (weak scaling, no
data-path collective); the step time is the max over ranks, and only the
headline section runs.
"""

from __future__ import annotations

import argparse
import json
import math
import os
from pathlib import Path
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = Path(__file__).resolve().parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

METRIC = "Mrays/s, 1M-tri 1080p; served p50/p99 latency vs plain path, same B200"
WIDTH, HEIGHT, SPP, BOUNCES = 1920, 1080, 4, 8
WORKLOAD = ("instanced PBR scene: 64 x 16,384-tri spheres + 2-tri ground + 1,024 emissive tris "
            "(1,049,602 tris), 1920x1080, 4 spp, 8 bounces, GGX+NEE, ReSTIR DI 32 candidates + "
            "1 temporal + 1 spatial (5 neighbours, r=30 px)")

# Algorithmic bytes per work unit of each stage (fixed figures, independent of
# the layout): ray 32 B, hit 20 B, path 36 B, material 32 B, shading triangle
# 72 B, shadow ray 44 B.
BYTES_PER_UNIT = {
    "raygen": 68.0,          # write ray 32 + path 36 per camera ray (in bounce-0 traversal)
    "trace_closest": 52.0,   # read ray 32, write hit 20 per ray
    "shade_hit": 304.0,      # read 32+20+36+32+36+36, write 36+32+44 per surface hit
    "shade_miss": 124.0,     # read ray 32 + hit 20 + path 36, write path 36
    "trace_shadow": 68.0,    # read shadow ray 44, read+write radiance 12+12
    "accumulate": 44.0,      # read radiance 12, read+write pixel 16+16
    "restir": 408.0,         # ray+hit 52, reservoir write 32, history read 32; spatial: ray+hit 52,
                             # 6 reservoir reads 192, write 32, selected sample 16
    "resolve": 40.0,         # read 24 B fixed-point sums, write 16 B pixel
    "sort": 104.0,           # key pass: read ray 32, write key 4; scatter: read key 4 + ray 32, write ray 32
}


def _peaks():
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU reference (oracle restatement of CpuReferenceRenderer), full renders of
# config 2 scaled for its brute-force intersector
# ---------------------------------------------------------------------------
# The CPU reference intersects every ray with every triangle in a Python loop
# over the triangles (renderers/reference/path_tracer.py:154-176): about 8
# rays/s at the headline scene's 1,049,602 triangles.  Its timed workload is
# therefore config 2 rescaled, rendered in full (camera and every extension
# segment of 8 bounces, its Lambert transport and CPU sky), never
# extrapolated; the CUDA renderer renders the same scene with the same
# transport in the `scaled_c2` section for the like-for-like ratio.
SCALED_C2 = dict(seed=5, instances=4, segments=32, bands=21, emitters=16, extent=4.0)
SCALED_C2_TRIANGLES = 4 * 1280 + 2 + 16
SCALED_C2_BOUNCES = 8
SCALED_C2_TILE = (48, 32)   # pixels one CPU process renders per step, 1 spp
SCALED_C2_WORKLOAD = ("config 2 scaled for the CPU reference's brute-force intersector: 4 instances of a "
                      "1,280-tri sphere + 2-tri ground + 16 emissive tris (5,138 tris), reference-compatible "
                      "transport (Lambert, CPU sky), 8 bounces, all closest-hit segments rendered")


def _cpu_scaled_worker(seed):
    """One full reference render (48x32, 1 spp, every bounce) of the scaled
    scene by the oracle restatement of CpuReferenceRenderer; returns
    (closest-hit rays, seconds)."""
    os.environ["OMP_NUM_THREADS"] = "1"
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["MKL_NUM_THREADS"] = "1"
    from oracle import reference_path_tracer as ref
    from ordinarylight_b200 import scenes

    scene, camera = scenes.instanced_spheres(**SCALED_C2)
    counter = ref.RayCounter()
    t0 = time.perf_counter()
    ref.render_frame(scene, camera, SCALED_C2_TILE[0], SCALED_C2_TILE[1], samples=1, max_bounces=SCALED_C2_BOUNCES,
                     seed=int(seed), counter=counter)
    return counter.rays, time.perf_counter() - t0


class CpuReference:
    """Pool of spawn workers, one per host core: a step is one full render of
    the scaled scene per process (distinct seeds), rays summed, the slowest
    process's time taken."""

    def __init__(self, processes=None):
        import multiprocessing as mp

        self.processes = processes or os.cpu_count() or 1
        self.pool = mp.get_context("spawn").Pool(self.processes)
        self.step = 0

    def run_step(self):
        seeds = [1000 + self.step * self.processes + k for k in range(self.processes)]
        self.step += 1
        results = self.pool.map(_cpu_scaled_worker, seeds)
        return sum(r for r, _ in results), max(t for _, t in results)

    def close(self):
        self.pool.close()
        self.pool.join()

    def describe(self, steps):
        w, h = SCALED_C2_TILE
        return (f"{SCALED_C2_WORKLOAD}: per step, one {w}x{h} render at 1 spp per process (camera rays and all "
                f"extension segments, counted as the reference's intersector sees them), {steps} step(s), one "
                f"process per core, slowest process timed; nothing extrapolated")


def cpu_reference_measure(steps, processes=None):
    ref = CpuReference(processes)
    try:
        total_rays, total_s = 0, 0.0
        for _ in range(steps):
            rays, secs = ref.run_step()
            total_rays += rays
            total_s += secs
        return total_rays / total_s / 1e6, ref.processes, ref.describe(steps)
    finally:
        ref.close()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = str(index)
        self.proc = None
        self.lines = []
        self.skip = 0    # samples taken before the timed region started

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-i", self.index, "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        # nvidia-smi takes a moment to start: wait for its first sample so
        # that the samples cover the whole timed region after this returns
        deadline = time.perf_counter() + 5.0
        while not self.lines and self.proc.poll() is None and time.perf_counter() < deadline:
            time.sleep(0.01)
        self.skip = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines[self.skip:]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# the CUDA arm
# ---------------------------------------------------------------------------
def _make_renderer(device):
    from ordinarylight_b200 import CudaWavefrontRenderer

    return CudaWavefrontRenderer(device=device, samples_per_pixel=SPP, max_bounces=BOUNCES, restir=True,
                                 restir_candidates=32, restir_temporal=True, restir_spatial=1,
                                 restir_neighbours=5, restir_radius=30.0)


def _profile(renderer):
    from ordinarylight_b200 import _native
    import ctypes

    count = ctypes.c_uint32()
    lib = renderer._lib
    _native.check(lib, renderer._ctx, lib.olc_frame_profile(renderer._ctx, None, 0, ctypes.byref(count)))
    records = (_native.OlcLaunchRecord * count.value)()
    _native.check(lib, renderer._ctx, lib.olc_frame_profile(renderer._ctx, records, count.value,
                                                            ctypes.byref(count)))
    return [(_native.STAGE_NAMES[r.stage], r.bounce, int(r.items), int(r.misses), float(r.ms)) for r in records]


def _launch_bytes(stage, bounce, items, misses):
    if stage == "trace_closest" and bounce == 0:
        # bounce-0 traversal generates its camera rays and their path records
        return (BYTES_PER_UNIT["raygen"] + BYTES_PER_UNIT["trace_closest"]) * items
    if stage == "shade":
        return BYTES_PER_UNIT["shade_hit"] * (items - misses) + BYTES_PER_UNIT["shade_miss"] * misses
    return BYTES_PER_UNIT[stage] * items


def _traffic_from_profiles(kernel):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    path = REPO / "profiles" / f"{kernel}_traffic.txt"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch_full_workload:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def run_ours(args, rank, world, device_index):
    import torch

    from ordinarylight_b200 import _native, scenes

    torch.cuda.set_device(device_index)
    scene, camera = scenes.instanced_spheres()
    renderer = _make_renderer(device_index)
    width, height = args.width, args.height
    out = torch.empty((height, width, 4), dtype=torch.float32, device=f"cuda:{device_index}")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device_index}")
    import ctypes

    handle = ctypes.c_void_p()
    _native.check(renderer._lib, renderer._ctx, renderer._lib.olc_stream(renderer._ctx, ctypes.byref(handle)))
    stream = torch.cuda.ExternalStream(handle.value, device=f"cuda:{device_index}")
    frame0 = 1000 * rank
    # warm-up: uploads the scene, builds its hierarchy and captures the frame's run into a CUDA graph,
    # which the timed frames replay
    for k in range(args.warmup):
        renderer.render_frame_into(scene, camera, width, height, out, frame_index=frame0 + k)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    clocks = ClockSampler(device_index)
    clocks.start()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    rays = 0
    stage_ms, stage_bytes, stage_launches = {}, {}, {}
    launches = 0
    torch.cuda.synchronize()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))  # evict L2 between timed steps
            starts[k].record(stream)
        renderer.render_frame_into(scene, camera, width, height, out, frame_index=frame0 + args.warmup + k)
        with torch.cuda.stream(stream):
            ends[k].record(stream)
        rays += renderer.last_timings["rays"]
        restir_records = 0
        for stage, bounce, items, misses, ms in _profile(renderer):
            stage_ms[stage] = stage_ms.get(stage, 0.0) + ms
            stage_bytes[stage] = stage_bytes.get(stage, 0.0) + _launch_bytes(stage, bounce, items, misses)
            stage_launches[stage] = stage_launches.get(stage, 0) + 1
            if stage == "restir":
                # per chunk two records: resampling (compaction, initial, one
                # spatial pass), then the reservoir samples' shadow-ray emission
                launches += 3 if restir_records % 2 == 0 else 1
                restir_records += 1
            else:
                launches += 3 if stage == "sort" else 1   # sort: keys, scan, scatter
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = sum(step_ms)
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{device_index}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        r = torch.tensor([float(rays)], dtype=torch.float64, device=f"cuda:{device_index}")
        dist.all_reduce(r, op=dist.ReduceOp.SUM)
        rays_all = float(r.item())
    else:
        rays_all = float(rays)
    value = rays_all / (total_ms * 1e3)

    # end to end through the public API: host output, per-step host clock
    e2e_steps = max(1, min(args.steps, 5))
    # page-locked output buffers come from a cache that warms up here; the
    # warm-up holds each frame while rendering the next, as the timed loop
    # does, so that both buffers the loop alternates between are cached
    img = None
    for k in range(2):
        img = renderer.render_frame(scene, camera, width, height, frame_index=frame0 + 490 + k)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_rays, h2d, d2h = 0, 0, 0
    for k in range(e2e_steps):
        img = renderer.render_frame(scene, camera, width, height, frame_index=frame0 + 500 + k)
        e2e_rays += renderer.last_timings["rays"]
        h2d += renderer.last_timings["h2d_bytes"]
        d2h += renderer.last_timings["d2h_bytes"]
    e2e_s = time.perf_counter() - t0
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{device_index}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
        r = torch.tensor([float(e2e_rays)], dtype=torch.float64, device=f"cuda:{device_index}")
        dist.all_reduce(r, op=dist.ReduceOp.SUM)
        e2e_rays = float(r.item())
    e2e = e2e_rays / e2e_s / 1e6
    finite = bool(np.all(np.isfinite(img)))
    timings = dict(renderer.last_timings)

    # dominant kernel roofline
    peak, peak_kind = _peaks()
    dominant = max(stage_ms, key=stage_ms.get)
    per_launch_bytes = stage_bytes[dominant] / stage_launches[dominant]
    per_launch_ms = stage_ms[dominant] / stage_launches[dominant]
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9
    stages = {name: {"ms_per_step": stage_ms[name] / args.steps,
                     "share": stage_ms[name] / sum(stage_ms.values()),
                     "achieved_gbs": stage_bytes[name] / (stage_ms[name] * 1e-3) / 1e9 if stage_ms[name] else 0.0}
              for name in stage_ms}
    renderer.close()
    if rank != 0:
        return None
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "Mrays/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded scene generators, ordinarylight_b200/scenes.py)",
        "config": {"workload": WORKLOAD if (width, height) == (WIDTH, HEIGHT) else
                   WORKLOAD.replace("1920x1080", f"{width}x{height} (reduced for profiling)"),
                   "width": width, "height": height, "spp": SPP, "max_bounces": BOUNCES,
                   "triangles": 1049602, "parallelism": f"replicas x{world} (independent frames per GPU)",
                   "l2": "256 MiB buffer written between timed steps (L2 flush); per-frame queues 1.7 GB"},
        "rays_per_step": rays_all / args.steps,
        "mrays_closest_hit": None,
        "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": h2d // e2e_steps,
                "d2h_bytes_per_step": d2h // e2e_steps, "steps": e2e_steps, "finite": finite},
        "roofline": {"kernel": dominant, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": _traffic_from_profiles(dominant),
                     "algorithmic_bytes_per_launch": per_launch_bytes, "ms_per_launch": per_launch_ms,
                     "limiter": ("dependent-load latency and SIMD divergence, not HBM: BVH traversal with the "
                                 "instanced scene's nodes in L2 (ncu: 2 MB of DRAM reads per 921,600 camera "
                                 "rays, 8-19 of 32 lanes active, ~3 long-scoreboard stalls per issue, "
                                 "ALU pipe 45-47 % of peak; "
                                 "profiles/hot_kernels_instanced_640x360.md)")
                     if dominant == "trace_closest" else None},
        "stages": stages,
        "gpu_launches": launches,
        "clocks": clock_info,
        "last_frame": {k: timings[k] for k in ("camera_rays", "extension_rays", "shadow_rays", "gpu_ms",
                                               "restir_history_used", "traversal_errors", "queue_overflow")},
    }
    cr = timings["camera_rays"] + timings["extension_rays"]
    line["mrays_closest_hit"] = cr * args.steps / (total_ms * 1e3) if world == 1 else None
    return line


# ---------------------------------------------------------------------------
# secondary sections (N = 1)
# ---------------------------------------------------------------------------
def _cpu_room_worker(args):
    seed, width, height, bounces = args
    os.environ["OMP_NUM_THREADS"] = "1"
    from oracle import reference_path_tracer as ref
    from ordinarylight_b200 import scenes

    scene, camera = scenes.box_room()
    counter = ref.RayCounter()
    t0 = time.perf_counter()
    ref.render_frame(scene, camera, width, height, samples=1, max_bounces=bounces, seed=seed, counter=counter)
    return counter.rays, time.perf_counter() - t0


def run_config1(device_index, processes=None):
    """Closed-box room, 256x256, 16 spp, 4 bounces, reference-compatible
    transport: closest-hit rays per second on the GPU against the CPU
    reference (oracle) on all host cores."""
    import multiprocessing as mp

    import torch

    from ordinarylight_b200 import CudaWavefrontRenderer, scenes

    scene, camera = scenes.box_room()
    with CudaWavefrontRenderer(device=device_index, mode="reference_compatible", samples_per_pixel=16,
                               max_bounces=4, seed=1) as r:
        for k in range(3):
            r.render_frame(scene, camera, 256, 256, frame_index=k)
        rays, gpu_ms, wall = 0, 0.0, 0.0
        for k in range(10):
            t0 = time.perf_counter()
            r.render_frame(scene, camera, 256, 256, frame_index=10 + k)
            wall += time.perf_counter() - t0
            rays += r.last_timings["closest_hit_rays"]
            gpu_ms += r.last_timings["gpu_ms"]
    torch.cuda.synchronize()
    processes = processes or os.cpu_count() or 1
    with mp.get_context("spawn").Pool(processes) as pool:
        res = pool.map(_cpu_room_worker, [(100 + k, 256, 256, 4) for k in range(processes)])
    cpu_rays = sum(r for r, _ in res)
    cpu_s = max(t for _, t in res)
    gpu = rays / (gpu_ms * 1e3)
    cpu = cpu_rays / cpu_s / 1e6
    return {"workload": "closed-box room (36 tris), 256x256, 16 spp, 4 bounces, reference-compatible transport",
            "gpu_mrays_closest_hit": gpu, "gpu_e2e_mrays_closest_hit": rays / wall / 1e6,
            "cpu_mrays_closest_hit": cpu, "cpu_cores": processes,
            "cpu_sample": f"{processes} processes x 256x256 at 1 spp, 4 bounces, slowest process timed",
            "gpu_over_cpu": gpu / cpu, "e2e_over_cpu": rays / wall / 1e6 / cpu}


def run_scaled_c2(device_index, steps=5):
    """The CPU reference's workload on the GPU: the scaled config-2 scene with
    the reference-compatible transport and 8 bounces, at 1920x1080 and 1 spp
    so that the device is filled; closest-hit rays per second (camera and
    extension segments, what the CPU reference's counter counts)."""
    import torch

    from ordinarylight_b200 import CudaWavefrontRenderer, scenes

    scene, camera = scenes.instanced_spheres(**SCALED_C2)
    with CudaWavefrontRenderer(device=device_index, mode="reference_compatible", samples_per_pixel=1,
                               max_bounces=SCALED_C2_BOUNCES, seed=1) as r:
        for k in range(3):
            r.render_frame(scene, camera, 1920, 1080, frame_index=k)
        rays, gpu_ms, wall = 0, 0.0, 0.0
        for k in range(steps):
            t0 = time.perf_counter()
            r.render_frame(scene, camera, 1920, 1080, frame_index=10 + k)
            wall += time.perf_counter() - t0
            rays += r.last_timings["closest_hit_rays"]
            gpu_ms += r.last_timings["gpu_ms"]
    torch.cuda.synchronize()
    return {"workload": SCALED_C2_WORKLOAD + "; GPU image 1920x1080 at 1 spp",
            "gpu_mrays_closest_hit": rays / (gpu_ms * 1e3), "gpu_e2e_mrays_closest_hit": rays / wall / 1e6}


def run_config3(device_index, steps=5):
    """Terrain (2048^2 fBm heightfield, 8,380,418 triangles) under a 128^3
    fBm volume (sigma_t scale 0.5, albedo 0.9), sky 1.0 + sun; 1280x720,
    8 spp, 6 bounces."""
    import torch

    from ordinarylight_b200 import CudaWavefrontRenderer, scenes

    scene, camera = scenes.terrain()
    with CudaWavefrontRenderer(device=device_index, samples_per_pixel=8, max_bounces=6, seed=1) as r:
        r.render_frame(scene, camera, 1280, 720, frame_index=0)
        first_upload_ms = r.last_timings["scene_upload_ms"]     # pack, copies and hierarchy build, first time
        first_build_ms = r.bvh_info()["build_ms"]
        warm_upload_ms = r._ensure_scene(scene, force=True)       # the same upload again, everything warm
        for k in range(1, 3):
            r.render_frame(scene, camera, 1280, 720, frame_index=k)
        rays, gpu_ms = 0, 0.0
        stage = {}
        for k in range(steps):
            r.render_frame(scene, camera, 1280, 720, frame_index=10 + k)
            rays += r.last_timings["rays"]
            gpu_ms += r.last_timings["gpu_ms"]
            for name, _b, _i, _m, ms in _profile(r):
                stage[name] = stage.get(name, 0.0) + ms / steps
        build_ms = r.bvh_info()["build_ms"]
    torch.cuda.synchronize()
    return {"workload": "terrain 2048^2 fBm heightfield (8,380,418 tris) + 128^3 fBm volume "
                        "(sigma_t 0.5, albedo 0.9, delta tracking), sky + sun, 1280x720, 8 spp, 6 bounces",
            "mrays_per_s": rays / (gpu_ms * 1e3), "ms_per_frame": gpu_ms / steps, "bvh_build_ms": build_ms,
            "first_upload_ms": first_upload_ms, "first_bvh_build_ms": first_build_ms,
            "warm_upload_ms": warm_upload_ms,
            "stage_ms_per_frame": stage}


def _plain_frames(device_index, requests, limit=None):
    """The plain per-request path as a user drives it: one renderer,
    ``render_frame`` per request (the scene is uploaded and its BVH built
    whenever it differs from the previous request's, as the reference's
    resident-scene cache does), bounce limit set by ``reconfigure``.
    Returns (service seconds per request, rays per request)."""
    from ordinarylight_b200 import CudaWavefrontRenderer

    service, rays = [], []
    with CudaWavefrontRenderer(device=device_index, restir=True, restir_candidates=32, restir_spatial=1,
                               restir_neighbours=5, restir_radius=30.0, seed=1) as r:
        for q in requests[:limit]:
            t0 = time.perf_counter()
            if q.max_bounces is not None and q.max_bounces != r.config.max_bounces:
                r.reconfigure(max_bounces=q.max_bounces)
            r.render_frame(q.scene, q.camera, q.width, q.height, samples=q.samples, frame_index=q.frame_index)
            service.append(time.perf_counter() - t0)
            rays.append(r.last_timings["rays"])
    return service, rays


def _fifo_latency_ms(arrivals, service):
    """Completion minus arrival of a single FIFO worker."""
    finish, lat = 0.0, []
    for at, sv in zip(arrivals, service):
        finish = max(finish, at) + sv
        lat.append((finish - at) * 1e3)
    return lat, finish - arrivals[0]


def run_batched(device_index, tune=True):
    """64 jobs over nine rescaled configuration scenes: one wavefront after
    the autotuner, against the same jobs one at a time, both through
    render_frame (scene uploads on change) and with every scene resident."""
    import torch

    from ordinarylight_b200 import CudaWavefrontRenderer, workloads
    from ordinarylight_b200.autotune import autotune
    from ordinarylight_b200.renderers.cuda import host_image

    variants = workloads.batch_scene_variants()
    requests = workloads.batch_requests(variants, 64, seed=4)
    outs = [host_image(r.height, r.width) for r in requests]
    frame_service, frame_rays = _plain_frames(device_index, requests)
    with CudaWavefrontRenderer(device=device_index, restir=True, restir_candidates=32, restir_spatial=1,
                               restir_neighbours=5, restir_radius=30.0, seed=1) as r:
        for v in variants:
            r.resident_scene(v[0])
        # one job per run, scenes resident; one untimed pass first so that
        # every job shape has its graph and the pixel arena its size, as the
        # batch below has after its warm-up
        for q, o in zip(requests, outs):
            r.render_batch([q], [o])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain_rays, plain_gpu = 0, 0.0
        for q, o in zip(requests, outs):
            r.render_batch([q], [o])
            plain_rays += r.last_timings["rays"]
            plain_gpu += r.last_timings["gpu_ms"]
        plain_wall = time.perf_counter() - t0
        tuned = None
        if tune:
            res = autotune(r, requests, repeats=1)
            tuned = {"chunk_paths": res.chunk_paths, "block_size": res.block_size, "trace_block": res.trace_block,
                     "stack_depth": res.stack_depth, "sort_rays": res.sort_rays, "trials": len(res.trials),
                     "best_s": res.seconds,
                     "trial_s": [(t[0]["chunk_paths"], t[0]["block_size"], t[0]["trace_block"], t[0]["stack_depth"],
                                  t[0]["sort_rays"], round(t[1], 4)) for t in res.trials]}
        r.render_batch(requests, outs)
        torch.cuda.synchronize()
        walls, rays, gpu = [], 0, 0.0
        for _ in range(3):
            t0 = time.perf_counter()
            r.render_batch(requests, outs)
            walls.append(time.perf_counter() - t0)
            rays = r.last_timings["rays"]
            gpu = r.last_timings["gpu_ms"]
        wall = min(walls)
    frame_mrays = sum(frame_rays) / sum(frame_service) / 1e6
    return {"workload": "64 jobs: configs 1-3 rescaled to 10k-4M tris (9 scenes), resolutions {128^2, 256^2, "
                        "512^2, 720p, 1080p}, spp {1, 4, 16}, seeded cameras",
            "paths": workloads.request_paths(requests),
            "mrays_per_s": rays / wall / 1e6, "gpu_mrays_per_s": rays / (gpu * 1e3), "batch_s": wall,
            "plain_frame_mrays_per_s": frame_mrays, "plain_frame_s": sum(frame_service),
            "speedup_vs_plain_frame": (rays / wall / 1e6) / frame_mrays,
            "plain_resident_mrays_per_s": plain_rays / plain_wall / 1e6,
            "plain_resident_gpu_mrays_per_s": plain_rays / (plain_gpu * 1e3), "plain_resident_s": plain_wall,
            "speedup_vs_plain_resident": (rays / wall) / (plain_rays / plain_wall),
            "tuned": tuned}


def run_served(device_index, rates, count, budget_bytes, chunk_paths, frame_limit=40):
    """Poisson request streams over 8 resident scenes, one per arrival rate:
    the continuous-batching server against the plain path serving the stream
    one request at a time in arrival order (the reference's serialised
    render_async worker), both through render_frame (scene uploads on
    change; the first `frame_limit` requests, whose measured service times
    give the FIFO latency at every rate) and with every scene resident (all
    requests, in real time on the same arrivals)."""
    import torch

    from ordinarylight_b200 import CudaWavefrontRenderer, workloads
    from ordinarylight_b200.serving import RenderServer, SerialServer, poisson_arrivals, run_stream

    variants = workloads.served_scene_variants()
    requests = workloads.served_requests(variants, count, seed=5)
    frame_service, frame_rays = _plain_frames(device_index, requests, frame_limit)
    results = []
    with CudaWavefrontRenderer(device=device_index, restir=True, restir_candidates=32, restir_spatial=1,
                               restir_neighbours=5, restir_radius=30.0, seed=1, chunk_paths=chunk_paths) as r:
        for v in variants:
            r.resident_scene(v[0])
        warm = workloads.served_requests(variants, 16, seed=99)
        r.render_batch(warm)
        # one-time costs of the serving path (graph captures, growth of the
        # pixel arena, the chunk tables and the light pools) are paid by a
        # warm-up stream at the highest rate, whose many requests in flight
        # grow every buffer to what the measured streams need
        warm_server = RenderServer(r, budget_bytes=budget_bytes).start()
        run_stream(warm_server, warm, poisson_arrivals(float(rates[0]), len(warm), seed=98))
        run_stream(warm_server, requests, poisson_arrivals(float(max(rates)), len(requests), seed=97))
        warm_server.stop()
        torch.cuda.synchronize()
        for rate in rates:
            rate = float(rate)
            arrivals = poisson_arrivals(rate, count, seed=6)
            frame_lat, frame_wall = _fifo_latency_ms(arrivals[:frame_limit], frame_service)
            frame_mrays = sum(frame_rays) / frame_wall / 1e6
            # plain with resident scenes, real time: one request at a time in
            # arrival order on a worker thread (SerialServer)
            serial = SerialServer(r).start()
            run_stream(serial, requests, arrivals)
            serial.stop()
            plain = serial.stats.summary()
            # served arm, same arrivals
            torch.cuda.synchronize()
            server = RenderServer(r, budget_bytes=budget_bytes).start()
            futures = run_stream(server, requests, arrivals)
            server.stop()
            summary = server.stats.summary()
            ok = sum(1 for f in futures if f.exception() is None)
            results.append({
                "workload": f"{count} requests, Poisson {rate:g} req/s, 8 resident scenes (10k-8.4M tris), "
                            "resolutions {256^2, 512^2, 720p, 1080p}, spp {1, 4, 16}, bounces {4, 8}, "
                            f"HBM budget {budget_bytes / 1e9:g} GB, chunk {chunk_paths} paths",
                "rate_req_s": rate, "requests": count, "completed": ok, "rejected": summary["rejected"],
                "failed": summary["failed"], "p50_ms": summary["p50_ms"], "p99_ms": summary["p99_ms"],
                "mean_ms": summary["mean_ms"], "throughput_req_s": summary["throughput_req_s"],
                "mrays_per_s": summary["mrays_per_s"], "steps": summary["steps"],
                "plain_frame": {"requests": frame_limit, "p50_ms": float(np.percentile(frame_lat, 50)),
                                "p99_ms": float(np.percentile(frame_lat, 99)),
                                "throughput_req_s": frame_limit / frame_wall, "mrays_per_s": frame_mrays,
                                "mean_service_ms": float(np.mean(frame_service) * 1e3)},
                "plain_resident": {"p50_ms": plain["p50_ms"], "p99_ms": plain["p99_ms"],
                                   "mean_ms": plain["mean_ms"], "throughput_req_s": plain["throughput_req_s"],
                                   "mrays_per_s": plain["mrays_per_s"], "gpu_mrays_per_s": plain["gpu_mrays_per_s"]},
                "speedup_mrays_vs_plain_frame": summary["mrays_per_s"] / frame_mrays,
                "speedup_mrays_vs_plain_resident": summary["mrays_per_s"] / plain["mrays_per_s"]})
    return results


def targets_summary(line):
    """The north star's ratios in one place (the batched/served >= 3x over the
    plain per-request path, config 1 >= 100x the CPU reference)."""
    t = {}
    c1 = line.get("config1")
    if c1:
        t["config1_gpu_over_cpu"] = c1["gpu_over_cpu"]
        t["config1_e2e_over_cpu"] = c1["e2e_over_cpu"]
        t["config1_required"] = 100.0
    c2 = line.get("scaled_c2")
    cpu = line.get("cpu_baseline")
    if c2 and cpu:
        t["scaled_c2_gpu_over_cpu"] = c2["gpu_mrays_closest_hit"] / cpu["value"]
    b = line.get("batched")
    if b:
        t["batched_speedup_vs_plain_frame"] = b["speedup_vs_plain_frame"]
        t["batched_speedup_vs_plain_resident"] = b["speedup_vs_plain_resident"]
    sv = line.get("served")
    if sv:
        t["served_rate_req_s"] = sv["rate_req_s"]
        t["served_speedup_vs_plain_frame"] = sv["speedup_mrays_vs_plain_frame"]
        t["served_speedup_vs_plain_resident"] = sv["speedup_mrays_vs_plain_resident"]
        t["served_p50_ms"] = sv["p50_ms"]
        t["served_p99_ms"] = sv["p99_ms"]
        t["served_rejected"] = sv["rejected"]
    if b or sv:
        t["systems_required"] = 3.0
    return t


def run_reference_arm(args):
    """The CPU reference's own implementation of the path (the oracle
    restatement of CpuReferenceRenderer) on all host cores, on the scaled
    config-2 workload, each step a full render per process."""
    steps = args.steps
    ref = CpuReference(args.cpu_processes)
    try:
        for _ in range(max(args.warmup, 1)):
            ref.run_step()
        total_rays, total_s = 0, 0.0
        for _ in range(steps):
            rays, secs = ref.run_step()
            total_rays += rays
            total_s += secs
    finally:
        ref.close()
    value = total_rays / total_s / 1e6
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "Mrays/s",
        "n_gpus": args.gpus,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": total_s * 1e3 / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded scene generators, ordinarylight_b200/scenes.py)",
        "config": {"workload": SCALED_C2_WORKLOAD, "width": SCALED_C2_TILE[0], "height": SCALED_C2_TILE[1],
                   "spp": 1, "max_bounces": SCALED_C2_BOUNCES, "triangles": SCALED_C2_TRIANGLES,
                   "parallelism": f"host cores x{ref.processes} (one render per process per step)",
                   "full_config_2": "the 1,049,602-triangle scene is beyond the brute-force intersector "
                                    "(about 8 rays/s); the CUDA line's scaled_c2 section renders this scaled "
                                    "scene with the same transport"},
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": ref.processes, "kind": "port",
                         "sample": ref.describe(steps)},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def main():
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--cpu-steps", type=int, default=1)
    p.add_argument("--cpu-processes", type=int, default=None)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--width", type=int, default=WIDTH, help="image width (a smaller case for profiling)")
    p.add_argument("--height", type=int, default=HEIGHT, help="image height (a smaller case for profiling)")
    p.add_argument("--sections", default="config1,scaled_c2,config3,batched,served",
                   help="secondary sections run at N=1 (comma list; empty for the headline alone)")
    p.add_argument("--served-rates", default="5,25,50,100,200",
                   help="Poisson arrival rates (req/s), ascending; the last is reported as `served`, all in "
                        "`served_sweep`")
    p.add_argument("--served-requests", type=int, default=150)
    p.add_argument("--served-budget-gb", type=float, default=150.0)
    p.add_argument("--served-chunk", type=int, default=1 << 23)
    args = p.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference_arm(args)), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device(f"cuda:{local}"))
    try:
        line = run_ours(args, rank, world, local)
        if rank == 0 and world == 1:
            sections = [x for x in args.sections.split(",") if x]
            if "config1" in sections:
                line["config1"] = run_config1(local, args.cpu_processes)
            if "scaled_c2" in sections:
                line["scaled_c2"] = run_scaled_c2(local)
            if "config3" in sections:
                line["config3"] = run_config3(local)
            if "batched" in sections:
                line["batched"] = run_batched(local)
            if "served" in sections:
                rates = [float(x) for x in args.served_rates.split(",") if x]
                sweep = run_served(local, rates, args.served_requests, args.served_budget_gb * 1e9,
                                   args.served_chunk)
                # the headline serving point: the highest swept rate, where the
                # plain path is far past its capacity and the server runs saturated
                line["served"] = sweep[-1]
                line["served_sweep"] = [{k: v[k] for k in ("rate_req_s", "p50_ms", "p99_ms", "throughput_req_s",
                                                          "mrays_per_s", "rejected", "completed",
                                                          "speedup_mrays_vs_plain_frame",
                                                          "speedup_mrays_vs_plain_resident", "plain_resident",
                                                          "plain_frame")} for v in sweep]
            if not args.no_cpu_baseline:
                value, cores, sample = cpu_reference_measure(args.cpu_steps, args.cpu_processes)
                line["cpu_baseline"] = {"value": value, "unit": "Mrays/s", "cores": cores, "kind": "port",
                                        "sample": sample,
                                        "workload": SCALED_C2_WORKLOAD + "; see scaled_c2 for the GPU's rate"}
            targets = targets_summary(line)
            if targets:
                # placed right after `config` so that a truncated log keeps it
                keys = list(line)
                at = keys.index("config") + 1
                line = {**{k: line[k] for k in keys[:at]}, "targets": targets, **{k: line[k] for k in keys[at:]}}
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
