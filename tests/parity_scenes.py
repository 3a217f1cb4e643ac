"""Scenes of the production-estimator parity tests, shared by the fixture
generator (tests/golden/make_production_golden.py) and the GPU tests.

* :func:`ggx_pair` — two 1,280-triangle spheres of one GGX material
  (roughness x metallic sweep) on a grey ground, lit by a one-sided quad
  emitter, a small tinted two-sided emitter triangle, a point light and the
  GPU shaders' analytic sky (no environment set).
* the closed-box room of ordinarylight_b200.scenes in production mode
  (GGX roughness 1, analytic sky through the open front).
* :func:`restir_spheres` — the 64-emitter instanced test scene of the ReSTIR
  tests, under a black environment.

Every case is rendered at CASES[name]["size"] with the transport settings
in CASES[name]; the oracle's fixture and the GPU render use the same ones.
"""

from __future__ import annotations

import numpy as np

from ordinarylight_b200 import scenes as _scenes
import ordinarylight_b200 as _ol


def ggx_pair(roughness: float, metallic: float, module=None):
    m = module or _ol
    scene = m.Scene()
    v, i, n = _scenes.uv_sphere(32, 21)
    sphere = scene.create_mesh(v, i, m.Material(), normals=n, name="sphere")
    scene.add_instances(
        sphere,
        [m.Transform.translation((-1.15, 1.0, 0.0)),
         m.Transform.translation((1.1, 0.8, 0.4)) @ m.Transform.scale(0.8)],
        materials=[m.Material(base_color=(0.9, 0.6, 0.3), roughness=roughness, metallic=metallic),
                   m.Material(base_color=(0.3, 0.7, 0.9), roughness=roughness, metallic=metallic)])
    g = 6.0
    scene.add_mesh(np.array([[-g, 0, -g], [-g, 0, g], [g, 0, g], [g, 0, -g]], np.float32),
                   np.array([[0, 1, 2], [0, 2, 3]], np.uint32),
                   m.Material(base_color=(0.5, 0.5, 0.5), roughness=0.7), name="ground")
    q = 0.6
    scene.add_mesh(np.array([[-q, 3.5, -q], [q, 3.5, -q], [q, 3.5, q], [-q, 3.5, q]], np.float32),
                   np.array([[0, 1, 2], [0, 2, 3]], np.uint32),
                   m.Material(base_color=(0.0, 0.0, 0.0), emission=(6.0, 5.5, 5.0)), name="panel")
    scene.add_mesh(np.array([[2.5, 0.3, -1.5], [3.0, 1.6, -1.0], [2.6, 0.4, -0.4]], np.float32),
                   np.array([[0, 1, 2]], np.uint32),
                   m.Material(base_color=(0.0, 0.0, 0.0), emission=(8.0, 2.0, 1.0), emission_two_sided=True),
                   name="tinted")
    scene.add_light(m.PointLight(position=(-2.0, 2.5, -2.5), color=(1.0, 0.9, 0.8), intensity=4.0))
    camera = m.PerspectiveCamera(position=(0.0, 2.2, -5.0), target=(0.0, 0.8, 0.0), vertical_fov_degrees=45.0)
    return scene, camera


def restir_spheres(module=None):
    m = module or _ol
    scene, camera = _scenes.instanced_spheres(m, seed=7, instances=8, segments=32, bands=17, emitters=64,
                                              extent=6.0)
    scene.set_environment(m.EnvironmentLight(color=(0.0, 0.0, 0.0), intensity=0.0))
    return scene, camera


SWEEP = [(r, mt) for mt in (0.0, 1.0) for r in (0.05, 0.5, 1.0)]

CASES = {
    "box_room": dict(size=(64, 64), max_bounces=5, rr_start=3, rr_min=0.1),
    **{f"ggx_r{r:g}_m{mt:g}": dict(size=(64, 64), max_bounces=4, rr_start=0, rr_min=0.1) for r, mt in SWEEP},
    "restir_spheres": dict(size=(64, 48), max_bounces=2, rr_start=0, rr_min=0.1),
}


def build(name: str, module=None):
    if name == "box_room":
        return _scenes.box_room(module)
    if name == "restir_spheres":
        return restir_spheres(module)
    for r, mt in SWEEP:
        if name == f"ggx_r{r:g}_m{mt:g}":
            return ggx_pair(r, mt, module)
    raise KeyError(name)
