"""Seeded request mixes of the batched and served forms.

* :func:`batch_scene_variants` / :func:`batch_requests` — the batched form:
  64 independent jobs, each one of the three configuration scenes (the
  closed-box room, the instanced PBR spheres, the terrain with its volume)
  rescaled to 10k-4M triangles; resolutions drawn uniformly from
  {128^2, 256^2, 512^2, 1280x720, 1920x1080}, samples from {1, 4, 16},
  seeded cameras, the configuration's own bounce limit (4, 8, 6).
* :func:`served_scene_variants` / :func:`served_requests` — the served form:
  8 resident scenes (configuration variants of 10k-8M triangles); each
  request draws a scene uniformly, a resolution from {256^2, 512^2, 720p,
  1080p}, samples from {1, 4, 16}, a bounce limit from {4, 8} and a seeded
  camera.  Arrivals are Poisson (``serving.poisson_arrivals``).

Scenes are built once per variant and shared by the requests that draw them,
the way resident scenes are shared by a server's requests.
"""

from __future__ import annotations

import math

import numpy as np

from . import scene as _scene_module
from . import scenes
from .renderers.cuda import RenderRequest

BATCH_RESOLUTIONS = ((128, 128), (256, 256), (512, 512), (1280, 720), (1920, 1080))
SERVED_RESOLUTIONS = ((256, 256), (512, 512), (1280, 720), (1920, 1080))
SAMPLES = (1, 4, 16)
CONFIG_BOUNCES = {"room": 4, "spheres": 8, "terrain": 6}


def _variant(kind, size, volume=False):
    """(scene, camera, kind, triangle count) of one rescaled configuration."""
    if kind == "room":
        # 10 * n^2 wall triangles + 26 box/emitter triangles
        n = max(1, int(round(math.sqrt(max(size - 26, 10) / 10.0))))
        scene, camera = scenes.box_room(tessellation=n)
        tris = 10 * n * n + 26
    elif kind == "spheres":
        instances = max(1, int(round(size / 16384)))
        scene, camera = scenes.instanced_spheres(seed=2 + instances, instances=instances,
                                                 emitters=min(1024, 16 * instances))
        tris = instances * 16384 + 2 + min(1024, 16 * instances)
    else:
        grid = max(8, int(round(math.sqrt(size / 2.0))) + 1)
        scene, camera = scenes.terrain(size=grid, volume=volume, volume_size=64 if grid < 1024 else 128)
        tris = 2 * (grid - 1) ** 2
    return scene, camera, kind, tris


def batch_scene_variants():
    """Nine variants: three per configuration across 10k-4M triangles."""
    return [
        _variant("room", 10_000), _variant("room", 100_000), _variant("room", 1_000_000),
        _variant("spheres", 16_384), _variant("spheres", 262_144), _variant("spheres", 4_194_304),
        _variant("terrain", 10_000, volume=True), _variant("terrain", 500_000, volume=True),
        _variant("terrain", 4_000_000, volume=True),
    ]


def served_scene_variants():
    """Eight resident scenes of 10k-8M triangles."""
    return [
        _variant("room", 10_000), _variant("room", 500_000),
        _variant("spheres", 16_384), _variant("spheres", 1_048_576), _variant("spheres", 4_194_304),
        _variant("terrain", 100_000, volume=True), _variant("terrain", 2_000_000, volume=False),
        _variant("terrain", 8_380_418, volume=True),
    ]


def seeded_camera(camera, rng, module=None):
    """The variant's camera orbited about its target by up to +-25 degrees
    and moved 0.85-1.15x its distance."""
    m = module or _scene_module
    pos = np.asarray(camera.position, np.float64)
    target = np.asarray(camera.target, np.float64)
    offset = pos - target
    angle = math.radians(rng.uniform(-25.0, 25.0))
    c, s = math.cos(angle), math.sin(angle)
    offset = np.array([c * offset[0] + s * offset[2], offset[1], -s * offset[0] + c * offset[2]])
    offset *= rng.uniform(0.85, 1.15)
    return m.PerspectiveCamera(position=tuple(float(x) for x in target + offset),
                               target=tuple(float(x) for x in target),
                               vertical_fov_degrees=float(camera.vertical_fov_degrees))


def batch_requests(variants, count=64, seed=4):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        scene, camera, kind, _ = variants[int(rng.integers(len(variants)))]
        w, h = BATCH_RESOLUTIONS[int(rng.integers(len(BATCH_RESOLUTIONS)))]
        spp = SAMPLES[int(rng.integers(len(SAMPLES)))]
        out.append(RenderRequest(scene, seeded_camera(camera, rng), w, h, samples=spp, frame_index=k,
                                 max_bounces=CONFIG_BOUNCES[kind]))
    return out


def served_requests(variants, count, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        scene, camera, _kind, _ = variants[int(rng.integers(len(variants)))]
        w, h = SERVED_RESOLUTIONS[int(rng.integers(len(SERVED_RESOLUTIONS)))]
        spp = SAMPLES[int(rng.integers(len(SAMPLES)))]
        bounces = (4, 8)[int(rng.integers(2))]
        out.append(RenderRequest(scene, seeded_camera(camera, rng), w, h, samples=spp, frame_index=k,
                                 max_bounces=bounces))
    return out


def request_paths(requests) -> int:
    return sum(int(r.width) * int(r.height) * int(r.samples or 1) for r in requests)


__all__ = ["batch_scene_variants", "served_scene_variants", "batch_requests", "served_requests",
           "seeded_camera", "request_paths"]
