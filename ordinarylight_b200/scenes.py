"""Seeded synthetic scenes of the benchmark configurations.

All generators use ``numpy.random.default_rng(seed)``; the scenes are built
through the public scene API (``Scene.add_mesh``/``create_mesh``/
``add_instances``), so they work with this package's scene model and with
the reference's ``ordinarylight.Scene`` (pass ``module=ordinarylight``).

* :func:`box_room` — closed-box room: 2x2x2 box of 5 quads (open front),
  two rotated inner boxes, 0.5x0.5 ceiling emitter of radiance (17, 12, 4);
  albedos 0.73 grey, 0.65 red, 0.12 green; fov 40.
* :func:`instanced_spheres` — 64 instances of a 16,384-triangle sphere with
  seeded transforms, a 2-triangle ground, GGX materials and 1,024 emissive
  triangles with log-uniform radiance in [1, 100].
* :func:`terrain` — fBm heightfield terrain (2048^2 grid) with sky and sun,
  optionally with a 128^3 fBm density volume.
"""

from __future__ import annotations

import math

import numpy as np

from . import scene as _scene_module

# Colours of the closed-box room (grey / red / green walls).
ROOM_WHITE = (0.73, 0.73, 0.73)
ROOM_RED = (0.65, 0.05, 0.05)
ROOM_GREEN = (0.12, 0.45, 0.15)
ROOM_LIGHT = (17.0, 12.0, 4.0)


def _quad(a, b, c, d):
    """Two triangles of the quad a-b-c-d (counter-clockwise seen from the
    side the normal faces)."""
    v = np.array([a, b, c, d], np.float32)
    i = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    return v, i


def _box(size):
    """Closed axis-aligned box centred at the origin (12 triangles, outward)."""
    sx, sy, sz = (s * 0.5 for s in size)
    v = np.array([[-sx, -sy, -sz], [sx, -sy, -sz], [sx, sy, -sz], [-sx, sy, -sz],
                  [-sx, -sy, sz], [sx, -sy, sz], [sx, sy, sz], [-sx, sy, sz]], np.float32)
    faces = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 4, 7, 3), (1, 2, 6, 5), (0, 1, 5, 4), (3, 7, 6, 2)]
    idx = []
    for a, b, c, d in faces:
        idx += [[a, b, c], [a, c, d]]
    return v, np.array(idx, np.uint32)


def _tessellate(quad, n):
    """Split the quad (4 vertices, 2 triangles) into an n x n grid of quads."""
    v, _ = quad
    a, b, c, d = (np.asarray(x, np.float64) for x in v)
    s = np.linspace(0.0, 1.0, n + 1)
    u, w = np.meshgrid(s, s, indexing="ij")
    pts = ((1 - u)[..., None] * (1 - w)[..., None] * a + u[..., None] * (1 - w)[..., None] * b
           + u[..., None] * w[..., None] * c + (1 - u)[..., None] * w[..., None] * d)
    grid = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    p0, p1, p2, p3 = grid[:-1, :-1], grid[1:, :-1], grid[1:, 1:], grid[:-1, 1:]
    idx = np.concatenate([np.stack([p0, p1, p2], -1).reshape(-1, 3), np.stack([p0, p2, p3], -1).reshape(-1, 3)])
    return pts.reshape(-1, 3).astype(np.float32), idx.astype(np.uint32)


def box_room(module=None, *, light=ROOM_LIGHT, tessellation=1):
    """The closed-box room (36 triangles: 10 walls, 24 inner boxes, 2 emitter).

    Returns (scene, camera).  Geometry: walls x in [-1, 1], y in [0, 2],
    z in [-1, 1], front (z = -1) open; the emitter quad hangs 1e-3 below the
    ceiling and faces down; the inner boxes stand on the floor, rotated
    about y by -18 and +15 degrees.  ``tessellation`` n > 1 splits each wall
    into n x n quads (10 n^2 wall triangles), the same room with more
    geometry for the rescaled variants of the batched and served workloads.
    """
    m = module or _scene_module
    scene = m.Scene()
    white = m.Material(base_color=ROOM_WHITE)
    red = m.Material(base_color=ROOM_RED)
    green = m.Material(base_color=ROOM_GREEN)
    walls = [
        (_quad((-1, 0, -1), (-1, 0, 1), (1, 0, 1), (1, 0, -1)), white, "floor"),
        (_quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1)), white, "ceiling"),
        (_quad((-1, 0, 1), (-1, 2, 1), (1, 2, 1), (1, 0, 1)), white, "back"),
        (_quad((-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1)), red, "left"),
        (_quad((1, 0, -1), (1, 0, 1), (1, 2, 1), (1, 2, -1)), green, "right"),
    ]
    if tessellation > 1:
        walls = [(_tessellate(q, int(tessellation)), mat, name) for q, mat, name in walls]
    for (v, i), mat, name in walls:
        scene.add_mesh(v, i, mat, name=name)
    short_v, short_i = _box((0.6, 0.6, 0.6))
    tall_v, tall_i = _box((0.6, 1.2, 0.6))
    short_xf = m.Transform.translation((0.35, 0.3, -0.3)) @ m.Transform.rotation((0, 1, 0), math.radians(-18.0))
    tall_xf = m.Transform.translation((-0.35, 0.6, 0.35)) @ m.Transform.rotation((0, 1, 0), math.radians(15.0))
    scene.add_mesh(short_v, short_i, white, transform=short_xf, name="short-box")
    scene.add_mesh(tall_v, tall_i, white, transform=tall_xf, name="tall-box")
    lv, li = _quad((-0.25, 1.999, -0.25), (0.25, 1.999, -0.25), (0.25, 1.999, 0.25), (-0.25, 1.999, 0.25))
    scene.add_mesh(lv, li, m.Material(base_color=(0.0, 0.0, 0.0), emission=tuple(light)), name="light")
    camera = m.PerspectiveCamera(position=(0.0, 1.0, -3.9), target=(0.0, 1.0, 0.0), vertical_fov_degrees=40.0)
    return scene, camera


def uv_sphere(segments=128, bands=65, radius=1.0):
    """Sphere with 2*segments*(bands-1) triangles (128 x 65 -> 16,384) and
    analytic normals."""
    vertices = [(0.0, radius, 0.0)]
    for b in range(1, bands):
        theta = math.pi * b / bands
        y = math.cos(theta) * radius
        r = math.sin(theta) * radius
        for s in range(segments):
            phi = 2.0 * math.pi * s / segments
            vertices.append((r * math.cos(phi), y, r * math.sin(phi)))
    vertices.append((0.0, -radius, 0.0))
    v = np.array(vertices, np.float32)
    idx = []
    ring = lambda b, s: 1 + (b - 1) * segments + (s % segments)  # noqa: E731
    for s in range(segments):
        idx.append((0, ring(1, s + 1), ring(1, s)))
    for b in range(1, bands - 1):
        for s in range(segments):
            a, bb, c, d = ring(b, s), ring(b, s + 1), ring(b + 1, s + 1), ring(b + 1, s)
            idx.append((a, bb, c))
            idx.append((a, c, d))
    last = len(vertices) - 1
    for s in range(segments):
        idx.append((last, ring(bands - 1, s), ring(bands - 1, s + 1)))
    n = v / np.linalg.norm(v, axis=1, keepdims=True)
    return v, np.array(idx, np.uint32), n.astype(np.float32)


def _random_rotation(rng):
    """Uniform random rotation (quaternion from three uniforms, Shoemake)."""
    u1, u2, u3 = rng.random(3)
    q = np.array([math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                  math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3)])
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def instanced_spheres(module=None, *, seed=2, instances=64, segments=128, bands=65, emitters=1024,
                      extent=20.0):
    """Instanced PBR scene: ``instances`` spheres of 2*segments*(bands-1)
    triangles (64 x 16,384 = 1,048,576 at the defaults), transforms with
    positions U[-extent, extent]^3, uniform random rotations and scale
    U[0.5, 2]; GGX roughness U(0.05, 1), metallic Bernoulli(0.3), albedo
    U(0.1, 0.9)^3; a 2-triangle ground; ``emitters`` one-sided emissive
    triangles (log-uniform radiance in [1, 100]).  Returns (scene, camera)."""
    m = module or _scene_module
    rng = np.random.default_rng(seed)
    scene = m.Scene()
    v, i, n = uv_sphere(segments, bands)
    sphere = scene.create_mesh(v, i, m.Material(), normals=n, name="sphere")
    transforms, materials = [], []
    for _ in range(instances):
        xf = np.eye(4, dtype=np.float32)
        scale = rng.uniform(0.5, 2.0)
        xf[:3, :3] = _random_rotation(rng) * scale
        xf[:3, 3] = rng.uniform(-extent, extent, 3)
        transforms.append(m.Transform(xf))
        materials.append(m.Material(base_color=tuple(float(c) for c in rng.uniform(0.1, 0.9, 3)),
                                    roughness=float(rng.uniform(0.05, 1.0)),
                                    metallic=float(rng.random() < 0.3)))
    scene.add_instances(sphere, transforms, materials=materials)
    g = 4.0 * extent
    gv, gi = _quad((-g, -extent - 2.0, -g), (-g, -extent - 2.0, g), (g, -extent - 2.0, g), (g, -extent - 2.0, -g))
    scene.add_mesh(gv, gi, m.Material(base_color=(0.5, 0.5, 0.5), roughness=0.8), name="ground")
    if emitters:
        tri = scene.create_mesh(np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]], np.float32),
                                np.array([[0, 2, 1]], np.uint32), m.Material(), name="emitter")
        et, em = [], []
        for _ in range(emitters):
            xf = np.eye(4, dtype=np.float32)
            xf[:3, :3] = _random_rotation(rng) * rng.uniform(0.5, 1.5)
            xf[:3, 3] = rng.uniform(-1.2 * extent, 1.2 * extent, 3)
            et.append(m.Transform(xf))
            radiance = math.exp(rng.uniform(math.log(1.0), math.log(100.0)))
            tint = rng.uniform(0.5, 1.0, 3)
            em.append(m.Material(base_color=(0.0, 0.0, 0.0),
                                 emission=tuple(float(radiance * c) for c in tint / tint.max())))
        scene.add_instances(tri, et, materials=em)
    camera = m.PerspectiveCamera(position=(0.0, 8.0, -3.2 * extent), target=(0.0, 0.0, 0.0),
                                 vertical_fov_degrees=40.0)
    return scene, camera


def fbm_heightfield(size, seed=3, octaves=8, amplitude=50.0, lacunarity=2.0, gain=0.5):
    """Seeded fractional Brownian motion on a size x size grid: the sum of
    ``octaves`` bilinearly-interpolated value-noise layers."""
    rng = np.random.default_rng(seed)
    h = np.zeros((size, size), np.float64)
    freq, amp, norm = 4.0, 1.0, 0.0
    coords = np.linspace(0.0, 1.0, size, endpoint=False)
    for _ in range(octaves):
        cells = int(math.ceil(freq)) + 2
        lattice = rng.uniform(-1.0, 1.0, (cells, cells))
        x = coords * freq
        x0 = np.floor(x).astype(int)
        t = x - x0
        t = t * t * (3.0 - 2.0 * t)
        a = lattice[x0][:, x0]
        b = lattice[x0][:, x0 + 1]
        c = lattice[x0 + 1][:, x0]
        d = lattice[x0 + 1][:, x0 + 1]
        ty, tx = t[:, None], t[None, :]
        h += amp * ((a * (1 - tx) + b * tx) * (1 - ty) + (c * (1 - tx) + d * tx) * ty)
        norm += amp
        freq *= lacunarity
        amp *= gain
    return (h / norm * amplitude).astype(np.float32)


def grid_mesh(heights, spacing=1.0):
    n = heights.shape[0]
    xs = (np.arange(n, dtype=np.float32) - (n - 1) / 2.0) * spacing
    gx, gz = np.meshgrid(xs, xs)
    v = np.stack([gx.ravel(), heights.ravel(), gz.ravel()], axis=1).astype(np.float32)
    r = np.arange(n - 1)
    a = (r[:, None] * n + r[None, :]).ravel()
    b, c, d = a + 1, a + n + 1, a + n
    idx = np.concatenate([np.stack([a, d, c], 1), np.stack([a, c, b], 1)]).astype(np.uint32)
    return v, idx


def fbm_volume(size=128, seed=4, octaves=5):
    """Seeded fBm density grid in [0, 1] (z, y, x)."""
    rng = np.random.default_rng(seed)
    d = np.zeros((size, size, size), np.float32)
    coords = np.linspace(0.0, 1.0, size, endpoint=False)
    freq, amp, norm = 3.0, 1.0, 0.0
    for _ in range(octaves):
        cells = int(math.ceil(freq)) + 2
        lattice = rng.uniform(0.0, 1.0, (cells, cells, cells)).astype(np.float32)
        x = coords * freq
        x0 = np.floor(x).astype(int)
        t = (x - x0).astype(np.float32)
        t = t * t * (3.0 - 2.0 * t)
        acc = np.zeros_like(d)
        for dz in (0, 1):
            wz = (t if dz else 1 - t)[:, None, None]
            for dy in (0, 1):
                wy = (t if dy else 1 - t)[None, :, None]
                for dx in (0, 1):
                    wx = (t if dx else 1 - t)[None, None, :]
                    acc += wz * wy * wx * lattice[np.ix_(x0 + dz, x0 + dy, x0 + dx)]
        d += amp * acc
        norm += amp
        freq *= 2.0
        amp *= 0.5
    d /= norm
    return np.clip((d - 0.35) * 2.5, 0.0, 1.0).astype(np.float32)


def terrain(module=None, *, size=2048, seed=3, volume=True, volume_size=128):
    """Terrain plus volume: a size x size fBm heightfield (2*(size-1)^2
    triangles; 8,380,418 at 2048), Lambertian albedo 0.4, constant sky 1.0
    and a directional sun; optionally a volume_size^3 fBm density box with
    sigma_t scale 0.5 and albedo 0.9.  Returns (scene, camera)."""
    m = module or _scene_module
    scene = m.Scene()
    spacing = 512.0 / size
    heights = fbm_heightfield(size, seed=seed)
    v, i = grid_mesh(heights, spacing)
    scene.add_mesh(v, i, m.Material(base_color=(0.4, 0.4, 0.4)), name="terrain")
    scene.set_environment(m.EnvironmentLight(color=(1.0, 1.0, 1.0), intensity=1.0))
    scene.add_light(m.DirectionalLight(direction=(-0.4, -1.0, 0.3), color=(1.0, 0.95, 0.85), intensity=3.0))
    if volume and hasattr(scene, "add_volume") and hasattr(m, "VolumeMaterial"):
        density = fbm_volume(volume_size, seed=seed + 1)
        xf = m.Transform.translation((-60.0, 20.0, -60.0)) @ m.Transform.scale(120.0)
        scene.add_volume(density, m.VolumeMaterial(sigma_t_scale=0.5, albedo=0.9), transform=xf, name="cloud")
    camera = m.PerspectiveCamera(position=(0.0, 120.0, -300.0), target=(0.0, 0.0, 0.0), vertical_fov_degrees=50.0)
    return scene, camera


__all__ = ["box_room", "instanced_spheres", "terrain", "uv_sphere", "fbm_heightfield", "fbm_volume", "grid_mesh"]
