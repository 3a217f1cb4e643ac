"""ORACLE — test infrastructure only, never part of the product path.

Python side of the CPU restatement of the reference GPU wavefront's
production transport (GGX + Lambert BSDF, next-event estimation of analytic
lights, area emitters and the environment with the reference's MIS weights,
Russian roulette); the estimator itself is ``oracle/transport.c``, compiled
by :func:`build` into ``oracle/_build/libolotransport.so``.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU legs may import this module.

The scene is flattened here through the reference's public ``Scene`` API,
independently of the CUDA renderer's packer:

* triangles: ``mesh.world_vertices[mesh.indices]`` of every visible mesh in
  scene order (the order of ``Scene.triangles``, scene/_core.py:2732-2753),
  shading normals ``mesh.world_normals[mesh.indices]``;
* materials: base colour, roughness, metallic, emission and the two-sided
  emission flag of each mesh's material (the fields of ``MaterialData``,
  shaders/transport_v1/types.glsl:5-19, that an untextured opaque surface
  uses);
* emitters: triangles whose emission has positive luminance
  (0.2126, 0.7152, 0.0722) and area above 1e-12, selected in proportion to
  area x luminance through a cumulative distribution
  (``Scene.emissive_triangle_data`` / ``emissive_light_weight``,
  scene/_core.py:2637-2753);
* analytic lights: directional, point and spot lights as
  ``analytic_light_data`` describes them (scene/_core.py:2578-2632): radiance
  colour x intensity, the range cut-off and the cosines of the cone angles;
* environment: none gives the GPU shaders' analytic sky, an
  ``EnvironmentLight`` without an image its constant colour x intensity.

Textured and transmissive materials, environment images and volumes are
outside this restatement (``NotImplementedError``).
"""

from __future__ import annotations

import ctypes
import math
import os
from pathlib import Path
import subprocess

import numpy as np

HERE = Path(__file__).resolve().parent
SOURCE = HERE / "transport.c"
LIBRARY = HERE / "_build" / "libolotransport.so"

NEE = 1
ENV_NEE = 2
INVALID_RESAMPLE = 4

_LUMINANCE = np.array([0.2126, 0.7152, 0.0722])


class _Scene(ctypes.Structure):
    _fields_ = [
        ("num_triangles", ctypes.c_int32), ("positions", ctypes.c_void_p), ("normals", ctypes.c_void_p),
        ("material", ctypes.c_void_p), ("num_materials", ctypes.c_int32), ("materials", ctypes.c_void_p),
        ("num_emitters", ctypes.c_int32), ("emitter_triangle", ctypes.c_void_p), ("emitter_cdf", ctypes.c_void_p),
        ("emitter_pdf", ctypes.c_void_p), ("total_power", ctypes.c_double), ("num_lights", ctypes.c_int32),
        ("lights", ctypes.c_void_p), ("env_kind", ctypes.c_int32), ("env_color", ctypes.c_float * 3),
    ]


class _Camera(ctypes.Structure):
    _fields_ = [
        ("projection", ctypes.c_int32), ("position", ctypes.c_float * 3), ("forward", ctypes.c_float * 3),
        ("right", ctypes.c_float * 3), ("up", ctypes.c_float * 3), ("scale_x", ctypes.c_float),
        ("scale_y", ctypes.c_float),
    ]


class _Params(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int32), ("height", ctypes.c_int32), ("x0", ctypes.c_int32), ("y0", ctypes.c_int32),
        ("win_w", ctypes.c_int32), ("win_h", ctypes.c_int32), ("samples", ctypes.c_int32),
        ("first_sample", ctypes.c_int32), ("max_bounces", ctypes.c_int32), ("rr_start", ctypes.c_int32),
        ("rr_min_survival", ctypes.c_float), ("flags", ctypes.c_uint32), ("seed", ctypes.c_uint64),
    ]


def build(force: bool = False) -> Path:
    """Compile transport.c (gcc, OpenMP) if the library is missing or stale."""
    LIBRARY.parent.mkdir(exist_ok=True)
    if force or not LIBRARY.exists() or LIBRARY.stat().st_mtime < SOURCE.stat().st_mtime:
        subprocess.run(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-o", str(LIBRARY), str(SOURCE), "-lm"],
                       check=True)
    return LIBRARY


_lib = None


def _library():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(build()))
        lib.olo_render.argtypes = [ctypes.POINTER(_Scene), ctypes.POINTER(_Camera), ctypes.POINTER(_Params),
                                   ctypes.c_void_p, ctypes.c_void_p]
        lib.olo_render.restype = ctypes.c_int
        lib.olo_trace.argtypes = [ctypes.POINTER(_Scene), ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        lib.olo_trace.restype = ctypes.c_int
        lib.olo_bsdf.argtypes = [ctypes.c_void_p] * 6
        lib.olo_bsdf.restype = None
        lib.olo_sample_bsdf.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                        ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p]
        lib.olo_sample_bsdf.restype = None
        _lib = lib
    return _lib


class FlatScene:
    """A scene flattened for the C estimator; keeps its arrays alive."""

    def __init__(self, scene):
        if tuple(getattr(scene, "visible_volumes", ())):
            raise NotImplementedError("the production oracle restates surface transport only")
        positions, normals, material_index, materials = [], [], [], []
        for mesh in scene.visible_meshes:
            m = mesh.material
            if float(getattr(m, "transmission", 0.0)) > 0.001:
                raise NotImplementedError("transmissive materials are outside the production oracle")
            for slot in ("base_color", "metallic_roughness", "emissive", "normal", "occlusion", "transmission"):
                if getattr(m, f"{slot}_texture", None) is not None:
                    raise NotImplementedError("textured materials are outside the production oracle")
            if not len(mesh.indices):
                continue
            positions.append(mesh.world_vertices[mesh.indices])
            normals.append(mesh.world_normals[mesh.indices])
            material_index.append(np.full(len(mesh.indices), len(materials), np.int32))
            materials.append([*m.base_color, m.roughness, m.metallic, *m.emission,
                              1.0 if m.emission_two_sided else 0.0, 0.0])
        if positions:
            self.positions = np.ascontiguousarray(np.concatenate(positions), np.float32)
            self.normals = np.ascontiguousarray(np.concatenate(normals), np.float32)
            self.material_index = np.ascontiguousarray(np.concatenate(material_index), np.int32)
        else:
            self.positions = np.zeros((0, 3, 3), np.float32)
            self.normals = np.zeros((0, 3, 3), np.float32)
            self.material_index = np.zeros(0, np.int32)
        self.materials = np.ascontiguousarray(np.asarray(materials, np.float32).reshape(-1, 10))
        # emitters: area x luminance power distribution
        tri = self.positions.astype(np.float64)
        area = 0.5 * np.linalg.norm(np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]), axis=1)
        lum = (self.materials[self.material_index, 5:8].astype(np.float64) @ _LUMINANCE
               if len(self.material_index) else np.zeros(0))
        emitting = np.flatnonzero((lum > 0.0) & (area > 1e-12))
        power = area[emitting] * lum[emitting]
        self.total_power = float(power.sum())
        self.emitter_triangle = np.ascontiguousarray(emitting, np.int32)
        self.emitter_pdf = np.ascontiguousarray(power / self.total_power if len(power) else power, np.float64)
        cdf = np.cumsum(self.emitter_pdf)
        if len(cdf):
            cdf[-1] = 1.0
        self.emitter_cdf = np.ascontiguousarray(cdf, np.float64)
        self.lights = np.ascontiguousarray(self._lights(scene), np.float32)
        env = getattr(scene, "environment", None)
        if env is None:
            self.env_kind, self.env_color = 0, (0.0, 0.0, 0.0)
        else:
            if getattr(env, "image", None) is not None:
                raise NotImplementedError("environment images are outside the production oracle")
            self.env_kind = 1
            self.env_color = tuple(float(c) * float(env.intensity) for c in env.color)

    @staticmethod
    def _lights(scene):
        rows = []
        for light in getattr(scene, "lights", ()):
            kind = type(light).__name__
            row = np.zeros(16, np.float64)
            radiance = np.asarray(light.color, np.float64) * float(light.intensity)
            row[7:10] = radiance
            if kind == "DirectionalLight":
                row[0] = 1.0
                row[4:7] = light.direction
            elif kind in ("PointLight", "SpotLight"):
                row[1:4] = light.position
                row[10] = 0.0 if light.range is None else float(light.range)
                if kind == "SpotLight":
                    row[0] = 2.0
                    row[4:7] = light.direction
                    row[11] = math.cos(light.inner_cone_angle)
                    row[12] = math.cos(light.outer_cone_angle)
            else:
                raise NotImplementedError(f"light type {kind}")
            rows.append(row)
        return np.asarray(rows, np.float64).reshape(-1, 16)

    def struct(self) -> _Scene:
        s = _Scene()
        s.num_triangles = len(self.material_index)
        s.positions = self.positions.ctypes.data
        s.normals = self.normals.ctypes.data
        s.material = self.material_index.ctypes.data
        s.num_materials = len(self.materials)
        s.materials = self.materials.ctypes.data
        s.num_emitters = len(self.emitter_triangle)
        s.emitter_triangle = self.emitter_triangle.ctypes.data
        s.emitter_cdf = self.emitter_cdf.ctypes.data
        s.emitter_pdf = self.emitter_pdf.ctypes.data
        s.total_power = self.total_power
        s.num_lights = len(self.lights)
        s.lights = self.lights.ctypes.data
        s.env_kind = self.env_kind
        s.env_color = (ctypes.c_float * 3)(*self.env_color)
        return s


def camera_struct(camera, width: int, height: int) -> _Camera:
    """The reference camera model (renderers/reference/path_tracer.py:110-151)."""
    position = np.asarray(camera.position, np.float64)
    forward = np.asarray(camera.target, np.float64) - position
    forward /= np.linalg.norm(forward)
    right = np.cross(forward, np.asarray(camera.up, np.float64))
    right /= np.linalg.norm(right)
    up = np.cross(right, forward)
    aspect = width / height
    c = _Camera()
    kind = type(camera).__name__
    if kind == "PanoramicCamera":
        c.projection = 2
        c.scale_x = math.radians(camera.horizontal_fov_degrees) * 0.5
        c.scale_y = math.radians(camera.vertical_fov_degrees) * 0.5
    elif kind == "OrthographicCamera":
        c.projection = 1
        c.scale_x = aspect * camera.vertical_size * 0.5
        c.scale_y = camera.vertical_size * 0.5
    else:
        c.projection = 0
        half = math.tan(math.radians(camera.vertical_fov_degrees) / 2.0)
        c.scale_x, c.scale_y = aspect * half, half
    c.position = (ctypes.c_float * 3)(*position)
    c.forward = (ctypes.c_float * 3)(*forward)
    c.right = (ctypes.c_float * 3)(*right)
    c.up = (ctypes.c_float * 3)(*up)
    return c


def render(scene, camera, width: int, height: int, *, samples: int, max_bounces: int, rr_start: int = 0,
           rr_min_survival: float = 0.05, nee: bool = True, env_nee: bool = True, resample_invalid: bool = False,
           seed: int = 1, first_sample: int = 0, window=None, threads: int | None = None):
    """Per-pixel sums and sums of squares of the radiance of
    ``samples`` independent paths per pixel; returns (mean, sem), each
    (h, w, 3) float64 over the window (x0, y0, w, h) (default: the image).
    sem is the standard error of the mean from the per-sample variance."""
    flat = scene if isinstance(scene, FlatScene) else FlatScene(scene)
    x0, y0, ww, wh = window if window is not None else (0, 0, width, height)
    if not (0 <= x0 and 0 <= y0 and ww > 0 and wh > 0 and x0 + ww <= width and y0 + wh <= height):
        raise ValueError("the window must lie inside the image")
    if samples < 1 or max_bounces < 1:
        raise ValueError("samples and max_bounces must be positive")
    p = _Params(width=width, height=height, x0=x0, y0=y0, win_w=ww, win_h=wh, samples=samples,
                first_sample=first_sample, max_bounces=max_bounces, rr_start=rr_start,
                rr_min_survival=rr_min_survival,
                flags=(NEE if nee else 0) | (ENV_NEE if env_nee else 0) | (INVALID_RESAMPLE if resample_invalid else 0),
                seed=int(seed) & 0xFFFFFFFFFFFFFFFF)
    total = np.zeros((wh, ww, 3), np.float64)
    total2 = np.zeros((wh, ww, 3), np.float64)
    s, c = flat.struct(), camera_struct(camera, width, height)
    previous = os.environ.get("OMP_NUM_THREADS")
    if threads is not None:
        os.environ["OMP_NUM_THREADS"] = str(int(threads))
    try:
        status = _library().olo_render(ctypes.byref(s), ctypes.byref(c), ctypes.byref(p), total.ctypes.data,
                                       total2.ctypes.data)
    finally:
        if threads is not None:
            if previous is None:
                os.environ.pop("OMP_NUM_THREADS", None)
            else:
                os.environ["OMP_NUM_THREADS"] = previous
    if status != 0:
        raise MemoryError("the oracle could not allocate its hierarchy")
    mean = total / samples
    var = np.maximum(total2 / samples - mean * mean, 0.0) * samples / max(samples - 1, 1)
    return mean, np.sqrt(var / samples)


def trace(scene, origins, directions, t_min=1e-4):
    """Closest hits of rays: (triangle index or -1, t)."""
    flat = scene if isinstance(scene, FlatScene) else FlatScene(scene)
    o = np.ascontiguousarray(origins, np.float32)
    d = np.ascontiguousarray(directions, np.float32)
    tri = np.zeros(len(o), np.int32)
    t = np.zeros(len(o), np.float64)
    s = flat.struct()
    if _library().olo_trace(ctypes.byref(s), len(o), o.ctypes.data, d.ctypes.data, float(t_min), tri.ctypes.data,
                            t.ctypes.data) != 0:
        raise MemoryError("the oracle could not allocate its hierarchy")
    return tri, t


def bsdf(material10, n, view, out):
    """(f rgb, pdf) of the restated BSDF for one direction pair."""
    m = np.ascontiguousarray(material10, np.float32)
    n, view, out = (np.ascontiguousarray(x, np.float64) for x in (n, view, out))
    f = np.zeros(3, np.float64)
    pdf = ctypes.c_double()
    _library().olo_bsdf(m.ctypes.data, n.ctypes.data, view.ctypes.data, out.ctypes.data, f.ctypes.data,
                        ctypes.byref(pdf))
    return f, pdf.value


def sample_bsdf(material10, n, incoming, u, *, resample_invalid=False, seed=1):
    """Weights f cos / pdf of the restated BSDF sampler for the draws u
    (k, 3): lobe choice, then the two direction draws."""
    m = np.ascontiguousarray(material10, np.float32)
    n, incoming = (np.ascontiguousarray(x, np.float64) for x in (n, incoming))
    u = np.ascontiguousarray(u, np.float64)
    out = np.zeros((len(u), 3), np.float64)
    _library().olo_sample_bsdf(m.ctypes.data, n.ctypes.data, incoming.ctypes.data, len(u), u.ctypes.data,
                               INVALID_RESAMPLE if resample_invalid else 0, int(seed), out.ctypes.data)
    return out


__all__ = ["FlatScene", "sample_bsdf", "build", "render", "trace", "bsdf", "camera_struct", "NEE", "ENV_NEE", "INVALID_RESAMPLE"]
