"""Pins of the production-transport oracle (oracle/transport.c,
oracle/production.py) on CPU, before it is trusted as the checker of the
CUDA renderer's production mode:

* its BSDF equals the independent numpy restatement (oracle/pbr.py) of the
  same GLSL (ordinaryshade_primary.glsl:541-581);
* BSDF sampling against solid-angle quadrature, after the reference's own
  known answer (tests/test_transport_gpu.py,
  test_rough_bsdf_sampling_matches_solid_angle_quadrature): the mean sampled
  weight f cos / pdf equals the hemispherical integral of f cos; the
  reference's resampling of reflections below the surface
  (lighting.glsl:238-241) overshoots it, which is why the default estimator
  ends such paths instead;
* the white furnace, after the reference's
  test_graph_metal_white_furnace_and_rough_glass: one bounce under a
  constant environment of 1 returns the surface's directional albedo (the
  integral of f cos by quadrature), and rough metal stays in the reference's
  range [0.85, 1.01] (single-scattering GGX loses energy);
* its three estimators of one image (full next-event estimation with the
  environment sampled, next-event estimation of emitters and lights only,
  BSDF sampling alone) agree: the MIS weights of each pair sum to one;
* its geometry reproduces the reference's own closest hits on the closed-box
  room (tests/golden/config1_primary.npz, made by running the reference);
* every production fixture is reproduced bit for bit on a window re-render,
  so the fixtures are this oracle's output.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import pbr, production
from oracle import reference_path_tracer as ref
import parity_scenes
import ordinarylight_b200 as ol
from ordinarylight_b200 import scenes


def _material(base, roughness, metallic, emission=(0, 0, 0)):
    return np.array([*base, roughness, metallic, *emission, 0.0, 0.0], np.float32)


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


@pytest.mark.parametrize("roughness,metallic", [(0.05, 0.0), (0.5, 0.0), (1.0, 0.0), (0.05, 1.0), (0.5, 1.0),
                                                (0.3, 0.6)])
def test_c_bsdf_equals_the_numpy_restatement(roughness, metallic):
    rng = np.random.default_rng(11)
    base = (0.7, 0.4, 0.2)
    n = np.array([0.0, 0.0, 1.0])
    views = _unit(rng, 64)
    views[:, 2] = np.abs(views[:, 2])
    outs = _unit(rng, 64)
    for v, o in zip(views, outs):
        f, pdf = production.bsdf(_material(base, roughness, metallic), n, v, o)
        np.testing.assert_allclose(f, pbr.pbr_evaluate(base, roughness, metallic, n, v, o), rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(pdf, max(float(pbr.pbr_pdf(base, roughness, metallic, n, v, o)), 0.0),
                                   rtol=1e-6, atol=1e-12)


def _quadrature(base, roughness, metallic, view, k=512):
    """Integral of f cos over the sphere by the midpoint rule in (z, phi),
    as the reference's test lays out its directions."""
    z = 1.0 - 2.0 * (np.arange(k) + 0.5) / k
    phi = 2.0 * np.pi * (np.arange(k) + 0.5) / k
    zz, pp = np.meshgrid(z, phi, indexing="ij")
    s = np.sqrt(1.0 - zz * zz)
    out = np.stack([s * np.cos(pp), s * np.sin(pp), zz], -1).reshape(-1, 3)
    n = np.broadcast_to([0.0, 0.0, 1.0], out.shape)
    v = np.broadcast_to(view, out.shape)
    f = pbr.pbr_evaluate(base, roughness, metallic, n, v, out)
    return (f * np.abs(out[:, 2:3]) * 4.0 * np.pi).mean(axis=0)


@pytest.mark.parametrize("roughness,metallic", [(0.6, 0.7), (1.0, 0.0), (0.5, 1.0)])
def test_bsdf_sampling_matches_solid_angle_quadrature(roughness, metallic):
    base = (0.7, 0.4, 0.2)
    view = np.array([0.6, 0.0, 0.8])
    integral = _quadrature(base, roughness, metallic, view)
    rng = np.random.default_rng(3)
    count = 1 << 18
    u = rng.random((count, 3))
    mat = _material(base, roughness, metallic)
    weights = production.sample_bsdf(mat, [0, 0, 1], -view, u)
    estimate = weights.mean(axis=0)
    se = weights.std(axis=0, ddof=1) / np.sqrt(count)
    assert np.all(np.abs(estimate - integral) <= 4.0 * se + 2e-3 * integral), (estimate, integral, se)
    # the reference's resampling of invalid reflections keeps the mixture pdf
    # for a direction drawn from the cosine lobe alone: biased upwards
    resampled = production.sample_bsdf(mat, [0, 0, 1], -view, u, resample_invalid=True)
    assert np.all(resampled.mean(axis=0) > integral)


def _floor_under_unit_sky(base, roughness, metallic, view_dir):
    """A huge floor of one material under a constant environment of 1, seen
    by a 1-degree camera along view_dir."""
    scene = ol.Scene()
    g = 1.0e4
    scene.add_mesh(np.array([[-g, 0, -g], [-g, 0, g], [g, 0, g], [g, 0, -g]], np.float32),
                   np.array([[0, 1, 2], [0, 2, 3]], np.uint32),
                   ol.Material(base_color=base, metallic=metallic, roughness=roughness))
    scene.set_environment(ol.EnvironmentLight(color=(1.0, 1.0, 1.0), intensity=1.0))
    eye = np.array([0.0, 1.0, 0.0])
    camera = ol.PerspectiveCamera(position=tuple(eye), target=tuple(eye + np.asarray(view_dir)),
                                  vertical_fov_degrees=1.0)
    return scene, camera


@pytest.mark.parametrize("base,roughness,metallic", [((1.0, 1.0, 1.0), 0.4, 1.0), ((0.9, 0.6, 0.3), 1.0, 0.0),
                                                     ((0.7, 0.4, 0.2), 0.6, 0.7)])
@pytest.mark.parametrize("env_nee", [False, True])
def test_one_bounce_under_a_unit_sky_is_the_directional_albedo(base, roughness, metallic, env_nee):
    """White-furnace known answer: under a constant environment of 1, one
    bounce off a surface returns its directional albedo, the hemispherical
    integral of f cos for the view direction (by quadrature), whether the
    environment is reached by BSDF sampling alone or also by next-event
    estimation with the reference's weight pair.  For rough metal it lies in
    the reference's furnace range [0.85, 1.01] (single-scattering GGX loses
    energy).  (Near roughness 0 this BSDF's D is capped by the 1e-6 floor of
    its denominator, so it reflects less than 1 there by definition.)"""
    from image_parity import oracle_image_se

    d = np.array([0.0, -0.6, 0.8])
    scene, camera = _floor_under_unit_sky(base, roughness, metallic, d)
    mean, sem = production.render(scene, camera, 4, 4, samples=8192, max_bounces=2, env_nee=env_nee)
    # the floor's normal is +y: rotate the view into the quadrature's +z frame
    view = -d / np.linalg.norm(d)
    expected = _quadrature(base, roughness, metallic, np.array([view[0], view[2], view[1]]), k=1024)
    got = mean.reshape(-1, 3).mean(axis=0)
    assert np.all(np.abs(got - expected) <= 4.0 * oracle_image_se(sem) + 2e-3 * expected), (got, expected)
    if metallic == 1.0:
        assert np.all((got >= 0.85) & (got <= 1.01))


@pytest.mark.parametrize("name", ["box_room", "ggx_r0.5_m1", "ggx_r0.05_m1"])
def test_the_oracles_estimators_agree(name):
    """Each estimator as 8 independent batches (seeds), so that the standard
    errors come from batch means: BSDF sampling of small emitters off a
    near-mirror is heavy-tailed, and its per-sample variance understates
    the noise."""
    from image_parity import batch_estimate, compare

    case = parity_scenes.CASES[name]
    scene, camera = parity_scenes.build(name)
    if name != "box_room":      # a delta light reaches no BSDF-sampled path
        for light in list(scene.lights):
            scene.lights.remove(light)
    w, h = 32, 32
    runs = {}
    full = dict(env_nee=case["env_nee"])
    for label, kw in (("full", full), ("no-env-nee", dict(env_nee=False)), ("bsdf", dict(nee=False))):
        batches = [production.render(scene, camera, w, h, samples=512, max_bounces=case["max_bounces"],
                                     rr_start=case["rr_start"], seed=1000 * k + len(label), **kw)[0]
                   for k in range(8)]
        runs[label] = batch_estimate(np.stack(batches))
    for label in ("no-env-nee", "bsdf"):
        compare(*runs["full"], *runs[label], tolerance=0.01, label=label)


def test_oracle_geometry_reproduces_the_reference_hits(golden):
    data = golden("config1_primary.npz")
    scene, camera = scenes.box_room()
    o, d = ref.camera_rays(camera, 256, 256, np.random.default_rng(1))
    o32, d32 = o.astype(np.float32), d.astype(np.float32)
    tri, t = production.trace(scene, o32, d32, t_min=1e-4)
    expected = data["triangle"].astype(np.int32)
    mismatch = tri != expected
    assert np.array_equal(tri < 0, expected < 0)
    # a differing index is only allowed on an exact tie in distance
    assert np.all(np.abs(t[mismatch] - data["t"][mismatch]) <= 1e-5 * np.abs(data["t"][mismatch]))
    assert mismatch.sum() <= 64


@pytest.mark.parametrize("name", list(parity_scenes.CASES))
def test_production_fixtures_are_this_oracles_output(golden, name):
    data = golden(f"production_{name}.npz")
    scene, camera = parity_scenes.build(name)
    w, h = int(data["width"]), int(data["height"])
    x0, y0 = w // 2 - 1, h // 3
    mean, _ = production.render(scene, camera, w, h, samples=int(data["samples"]),
                                max_bounces=int(data["max_bounces"]), rr_start=int(data["rr_start"]),
                                rr_min_survival=float(data["rr_min"]), env_nee=bool(data["env_nee"]),
                                seed=int(data["seed"]), window=(x0, y0, 3, 2))
    assert mean.astype(np.float32).tobytes() == data["mean"][y0:y0 + 2, x0:x0 + 3].tobytes()
