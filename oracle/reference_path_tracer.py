"""ORACLE — test infrastructure only, never part of the product path.

CPU restatement (numpy) of OrdinaryLight's reference renderer,
``CpuReferenceRenderer`` -> ``ReferencePathTracer.render_hdr``
(ordinarylight/renderers/reference/cpu.py:58-68,
ordinarylight/renderers/reference/path_tracer.py:31-211).  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline/reference arm may
import it, as the checker and the timed CPU baseline.

Pinned: ``tests/golden/make_golden.py`` runs the reference itself and records
camera rays, closest-hit results and small rendered images; the CPU tests
require this restatement to reproduce them bit for bit.

The algorithm, in the reference's order of random draws (the sequence
matters for bit-exactness):

* per sample: camera rays with two ``rng.random((h, w), float32)`` jitter
  arrays (x then y), directions normalised in float64
  (path_tracer.py:110-151);
* per bounce, for the still-active rays: Moller-Trumbore against every
  triangle in packed order, ``|det| > 1e-7``, ``u, v >= 0``, ``u + v <= 1``,
  ``t > 1e-4``, strict ``<`` so the lowest index wins ties
  (path_tracer.py:154-176);
* miss: sky gradient (or constant/equirect environment) times throughput,
  path ends (path_tracer.py:67-72, :185-202);
* hit: emission times throughput, throughput *= albedo, origin moves
  1e-4 along the normal flipped against the ray, new direction
  normalize(n + s) with s a normalised ``rng.normal`` vector flipped into
  the hemisphere (path_tracer.py:74-87, :205-211);
* volumes: after each intersection, every active segment up to its hit
  (or unbounded for a miss) crosses the visible volumes' emission–absorption
  ray march (oracle/reference_volume.py, path_tracer.py:55-65): radiance +=
  throughput * volume radiance, throughput *= volume transmittance;
* average over samples, alpha 0 (path_tracer.py:89-95).
"""

from __future__ import annotations

import math

import numpy as np

from . import reference_volume

__all__ = ["ReferencePathTracer", "render_hdr", "camera_rays", "intersect", "RayCounter"]


class RayCounter:
    """Counts rows passed to ``intersect`` (closest-hit segments)."""

    def __init__(self):
        self.rays = 0
        self.calls = 0


def camera_rays(camera, width, height, rng):
    """Primary rays of one sample (path_tracer.py:110-151)."""
    position = np.asarray(camera.position, dtype=np.float32)
    forward = np.asarray(camera.target, dtype=np.float32) - position
    forward /= np.linalg.norm(forward)
    right = np.cross(forward, np.asarray(camera.up, dtype=np.float32))
    right /= np.linalg.norm(right)
    up = np.cross(right, forward)
    ys, xs = np.mgrid[0:height, 0:width]
    jitter_x = rng.random((height, width), dtype=np.float32)
    jitter_y = rng.random((height, width), dtype=np.float32)
    ndc_x = (xs + jitter_x) / width * 2.0 - 1.0
    ndc_y = 1.0 - (ys + jitter_y) / height * 2.0
    aspect = width / height
    kind = type(camera).__name__
    if kind == "PanoramicCamera":
        yaw = ndc_x * math.radians(camera.horizontal_fov_degrees) * 0.5
        pitch = ndc_y * math.radians(camera.vertical_fov_degrees) * 0.5
        cp = np.cos(pitch)[..., None]
        directions = (cp * np.cos(yaw)[..., None] * forward + cp * np.sin(yaw)[..., None] * right
                      + np.sin(pitch)[..., None] * up).reshape((-1, 3))
        origins = np.repeat(position[None, :], len(directions), axis=0)
    elif kind == "OrthographicCamera":
        half = camera.vertical_size * 0.5
        origins = (position[None, None, :] + ndc_x[..., None] * (aspect * half) * right
                   + ndc_y[..., None] * half * up).reshape((-1, 3))
        directions = np.repeat(forward[None, :], len(origins), axis=0)
    else:
        half = math.tan(math.radians(camera.vertical_fov_degrees) / 2.0)
        directions = (forward[None, None, :] + ndc_x[..., None] * (aspect * half) * right
                      + ndc_y[..., None] * half * up).reshape((-1, 3))
        origins = np.repeat(position[None, :], len(directions), axis=0)
    directions /= np.linalg.norm(directions, axis=1, keepdims=True)
    return origins, directions


def intersect(origins, directions, triangles, counter: RayCounter | None = None):
    """Closest hit by brute force over the packed triangles
    (path_tracer.py:154-176).  Returns (t, triangle index or -1)."""
    if counter is not None:
        counter.rays += len(origins)
        counter.calls += 1
    count = len(origins)
    best_t = np.full(count, np.inf, dtype=np.float32)
    best = np.full(count, -1, dtype=np.int32)
    for index, tri in enumerate(triangles):
        e1 = tri[1] - tri[0]
        e2 = tri[2] - tri[0]
        p = np.cross(directions, e2)
        det = p @ e1
        ok = np.abs(det) > 1e-7
        inv = np.zeros_like(det)
        inv[ok] = 1.0 / det[ok]
        s = origins - tri[0]
        u = np.sum(s * p, axis=1) * inv
        q = np.cross(s, e1)
        v = np.sum(directions * q, axis=1) * inv
        t = (q @ e2) * inv
        hit = ok & (u >= 0.0) & (v >= 0.0) & (u + v <= 1.0) & (t > 1e-4)
        nearer = hit & (t < best_t)
        best_t[nearer] = t[nearer]
        best[nearer] = index
    return best_t, best


def _normals(tris):
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    return n


def sky(directions, environment=None):
    """Environment or CPU sky gradient (path_tracer.py:185-202)."""
    if environment is not None:
        radiance = np.ones((len(directions), 3), np.float32)
        if environment.image is not None:
            lon = np.arctan2(directions[:, 2], directions[:, 0]) + environment.rotation
            u = np.mod(lon / (2.0 * np.pi) + 0.5, 1.0)
            v = np.arccos(np.clip(directions[:, 1], -1.0, 1.0)) / np.pi
            h, w, _c = environment.image.shape
            x = np.minimum((u * w).astype(np.int64), w - 1)
            y = np.minimum((v * h).astype(np.int64), h - 1)
            radiance = environment.image[y, x]
        return radiance * np.asarray(environment.color, np.float32) * float(environment.intensity)
    blend = np.clip(0.5 * (directions[:, 1] + 1.0), 0.0, 1.0)[:, None]
    return (1.0 - blend) * np.array((0.8, 0.8, 0.8)) + blend * np.array((0.2, 0.4, 0.9))


def cosine_hemisphere(normals, rng):
    """normalize(n + s), s uniform on the sphere flipped into n's hemisphere
    (path_tracer.py:205-211)."""
    s = rng.normal(size=normals.shape).astype(np.float32)
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    s[np.sum(s * normals, axis=1) < 0.0] *= -1.0
    d = normals + s
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d


def render_hdr(scene, camera, width, height, samples=1, max_bounces=3, seed=1, counter=None):
    """(height, width, 4) float32 linear HDR, alpha 0."""
    if width <= 0 or height <= 0:
        raise ValueError("width and height must be positive")
    if samples <= 0 or max_bounces <= 0:
        raise ValueError("samples and max_bounces must be positive")
    volumes = tuple(getattr(scene, "visible_volumes", ()))
    lights = tuple(getattr(scene, "lights", ()))
    triangles, colors, emissions = scene.triangles()
    rng = np.random.default_rng(seed)
    accumulated = np.zeros((height * width, 3), dtype=np.float32)
    env = getattr(scene, "environment", None)
    for _ in range(samples):
        origins, directions = camera_rays(camera, width, height, rng)
        radiance = np.zeros_like(origins)
        throughput = np.ones_like(origins)
        active = np.ones(len(origins), dtype=bool)
        for _bounce in range(max_bounces):
            ids = np.flatnonzero(active)
            if not len(ids):
                break
            hit_t, hit_tri = intersect(origins[ids], directions[ids], triangles, counter)
            if volumes:
                # every segment crosses the media first (path_tracer.py:55-65)
                entries, exits = reference_volume.intersect_unit_boxes(origins[ids], directions[ids], volumes)
                vol_rad, vol_t = reference_volume.integrate_volumes(volumes, origins[ids], directions[ids], entries,
                                                                    exits, max_distance=hit_t, lights=lights)
                radiance[ids] += throughput[ids] * vol_rad
                throughput[ids] *= vol_t[:, None]
            missed = hit_tri < 0
            if np.any(missed):
                rid = ids[missed]
                radiance[rid] += throughput[rid] * sky(directions[rid], env)
                active[rid] = False
            hit = ~missed
            if not np.any(hit):
                continue
            rid = ids[hit]
            tid = hit_tri[hit]
            points = origins[rid] + directions[rid] * hit_t[hit, None]
            normals = _normals(triangles[tid])
            flip = np.sum(normals * directions[rid], axis=1) > 0.0
            normals[flip] *= -1.0
            radiance[rid] += throughput[rid] * emissions[tid]
            throughput[rid] *= colors[tid]
            origins[rid] = points + normals * 1e-4
            directions[rid] = cosine_hemisphere(normals, rng)
        accumulated += radiance
    rgb = accumulated.reshape((height, width, 3)) / samples
    out = np.empty((height, width, 4), dtype=np.float32)
    out[..., :3] = rgb
    out[..., 3] = 0.0
    return out


class ReferencePathTracer:
    """Same surface as the reference class: ``ReferencePathTracer(seed)``."""

    def __init__(self, seed=1):
        self.seed = seed
        self.counter = RayCounter()

    def render_hdr(self, scene, camera, width, height, samples=1, max_bounces=3):
        return render_hdr(scene, camera, width, height, samples, max_bounces, self.seed, self.counter)


def render_frame(scene, camera, width, height, *, samples=1, max_bounces=3, seed=1, frame_index=0, counter=None):
    """CpuReferenceRenderer.render_frame: seed = config.seed + frame_index
    (cpu.py:58-68)."""
    return render_hdr(scene, camera, width, height, samples, max_bounces, seed + int(frame_index), counter)
