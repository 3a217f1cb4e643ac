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

# env_nee: whether the oracle also samples the environment at surface
# vertices.  Its estimator is the reference's (a cosine-hemisphere direction
# with the constant weight 1/2 against BSDF-sampled sky): unbiased, but on a
# near-mirror the cosine directions almost never meet the lobe and its noise
# is some twenty times that of BSDF sampling, so those fixtures leave the sky
# to BSDF sampling alone.
CASES = {
    "box_room": dict(size=(64, 64), max_bounces=5, rr_start=3, rr_min=0.1, env_nee=True),
    **{f"ggx_r{r:g}_m{mt:g}": dict(size=(64, 64), max_bounces=4, rr_start=0, rr_min=0.1, env_nee=r >= 0.5)
       for r, mt in SWEEP},
    "restir_spheres": dict(size=(64, 48), max_bounces=2, rr_start=0, rr_min=0.1, env_nee=True),
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


# ---------------------------------------------------------------------------
# Reference-compatible parity scenes: rendered by the reference's own
# CpuReferenceRenderer for the goldens (tests/golden/make_volume_golden.py)
# and by the CUDA renderer's reference-compatible mode in the GPU tests.
# ---------------------------------------------------------------------------
def _fbm_field(size, seed):
    return _scenes.fbm_volume(size, seed=seed, octaves=3)


def volume_room(module=None):
    """The closed-box room with two overlapping volumes that exercise every
    part of the reference's volume model: an emissive, scattering medium
    (Henyey-Greenstein phase, two scattering orders, a clip plane) lit by a
    point light with a range, a directional and a spot light, and a second
    medium with missing data, a mirrored nearest-neighbour transfer function
    and a log value mapping."""
    m = module or _ol
    scene, camera = _scenes.box_room(m)
    a = _fbm_field(12, 21)
    tf_a = m.Texture1D(np.array([[0.0, 0.0, 0.0, 0.0], [1.0, 0.5, 0.2, 0.3], [0.4, 0.6, 1.0, 0.9]], np.float32))
    mat_a = m.VolumeMaterial(transfer_function=tf_a, density_scale=0.8, emission_scale=0.5, step_size=0.05,
                             scattering_scale=1.0, scattering_color=(1.0, 0.9, 0.8),
                             phase_function="henyey_greenstein", anisotropy=0.3, scattering_albedo=(0.9, 0.8, 0.7),
                             scattering_orders=2)
    scene.add_volume(a, mat_a, transform=m.Transform.translation((-0.7, 0.2, -0.6)) @ m.Transform.scale(1.0),
                     clip_planes=((0.0, 1.0, 0.0, 0.35),), name="glow")
    b = _fbm_field(10, 22) + 0.05
    b[2:4, 3:6, 1:3] = np.nan
    tf_b = m.Texture1D(np.array([[0.0, 0.0, 0.0, 0.0], [0.2, 0.9, 0.3, 0.6], [0.9, 0.9, 0.9, 0.2],
                                 [0.1, 0.1, 0.8, 0.8]], np.float32), address_mode="mirror", linear_filter=False)
    mat_b = m.VolumeMaterial(transfer_function=tf_b, density_scale=0.6, emission_scale=0.8, step_size=0.04)
    scene.add_volume(b, mat_b, transform=m.Transform.translation((-0.25, 0.45, -0.35)) @ m.Transform.scale(0.8),
                     value_mapping="log", value_range=(0.05, 1.05), missing_data=True, name="mist")
    scene.add_light(m.PointLight(position=(0.0, 1.7, -0.4), color=(1.0, 0.9, 0.7), intensity=2.0, range=2.5))
    scene.add_light(m.DirectionalLight(direction=(0.3, -1.0, 0.4), color=(0.6, 0.7, 1.0), intensity=0.5))
    scene.add_light(m.SpotLight(position=(0.8, 1.5, -0.8), direction=(-0.6, -0.8, 0.5), color=(1.0, 0.4, 0.4),
                                intensity=3.0, inner_cone_angle=0.3, outer_cone_angle=0.7))
    return scene, camera


def scaled_instanced(module=None):
    """Config 2 scaled for the reference's brute-force intersector: 4
    instances of a 1,280-triangle sphere, 16 emissive triangles, the ground
    (5,138 triangles)."""
    m = module or _ol
    return _scenes.instanced_spheres(m, seed=5, instances=4, segments=32, bands=21, emitters=16, extent=4.0)


def scaled_terrain(module=None):
    """Config 3 scaled likewise: a 32 x 32 fBm heightfield (1,922 triangles)
    under a constant sky and a sun, with a 24^3 fBm medium in the reference's
    volume model (absorbing, faintly emissive, sun-lit single scattering with
    a second order)."""
    m = module or _ol
    scene = m.Scene()
    heights = _scenes.fbm_heightfield(32, seed=3)
    v, i = _scenes.grid_mesh(heights, 16.0)
    scene.add_mesh(v, i, m.Material(base_color=(0.4, 0.4, 0.4)), name="terrain")
    scene.set_environment(m.EnvironmentLight(color=(1.0, 1.0, 1.0), intensity=1.0))
    scene.add_light(m.DirectionalLight(direction=(-0.4, -1.0, 0.3), color=(1.0, 0.95, 0.85), intensity=3.0))
    tf = m.Texture1D(np.array([[0.0, 0.0, 0.0, 0.0], [0.3, 0.3, 0.35, 0.4], [0.1, 0.1, 0.1, 0.9]], np.float32))
    mat = m.VolumeMaterial(transfer_function=tf, density_scale=0.5, emission_scale=0.2, step_size=10.0,
                           scattering_scale=0.3, scattering_albedo=(0.9, 0.9, 0.9), scattering_orders=2)
    scene.add_volume(_fbm_field(24, 4), mat, transform=m.Transform.translation((-60.0, 20.0, -60.0))
                     @ m.Transform.scale(120.0), name="cloud")
    camera = m.PerspectiveCamera(position=(0.0, 120.0, -300.0), target=(0.0, 0.0, 0.0), vertical_fov_degrees=50.0)
    return scene, camera


COMPAT_CASES = {
    "scaled_instanced": dict(builder=scaled_instanced, size=(48, 32), max_bounces=4),
    "scaled_terrain": dict(builder=scaled_terrain, size=(48, 32), max_bounces=4),
}
