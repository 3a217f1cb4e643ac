"""GPU transport checks beyond the CPU reference's Lambert model: analytic
known answers (closed-box furnace; one directional or point light on a
GGX surface, evaluated by the oracle's restatement of the reference GPU
BSDF) and unbiasedness checks (next-event estimation with MIS against pure
BSDF sampling; ReSTIR DI against plain NEE)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import pbr, products
from oracle import reference_path_tracer as ref
from ordinarylight_b200 import CudaWavefrontRenderer, scenes
import ordinarylight_b200 as ol

pytestmark = pytest.mark.gpu


def _closed_box(emission, albedo):
    scene = ol.Scene()
    v = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float32)
    faces = [(0, 1, 2, 3), (4, 7, 6, 5), (0, 3, 7, 4), (1, 5, 6, 2), (0, 4, 5, 1), (3, 2, 6, 7)]
    idx = np.array([t for a, b, c, d in faces for t in ((a, b, c), (a, c, d))], np.uint32)
    scene.add_mesh(v, idx, ol.Material(base_color=albedo, emission=emission, emission_two_sided=True))
    camera = ol.PerspectiveCamera(position=(0.1, 0.2, -0.5), target=(0.3, -0.1, 1.0), vertical_fov_degrees=60.0)
    return scene, camera


def test_closed_box_furnace_has_the_analytic_radiance(native_library, cuda_device):
    """Inside a closed box whose walls all emit E with albedo a, every path
    collects E (1 + a + ... + a^(B-1)) — no variance at all."""
    emission, albedo, bounces = (0.5, 1.0, 2.0), (0.6, 0.6, 0.6), 4
    scene, camera = _closed_box(emission, albedo)
    expected = np.asarray(emission) * (1.0 - 0.6 ** bounces) / (1.0 - 0.6)
    with CudaWavefrontRenderer(mode="reference_compatible", max_bounces=bounces, samples_per_pixel=4) as r:
        img = r.render_frame(scene, camera, 32, 24)
    np.testing.assert_allclose(img[..., :3], np.broadcast_to(expected, img[..., :3].shape), rtol=2e-5)
    cpu = ref.render_hdr(scene, camera, 8, 6, samples=2, max_bounces=bounces, seed=1)
    np.testing.assert_allclose(cpu[..., :3], np.broadcast_to(expected, cpu[..., :3].shape), rtol=2e-5)


def _floor_scene(light):
    scene = ol.Scene()
    v = np.array([[-100, 0, -100], [-100, 0, 100], [100, 0, 100], [100, 0, -100]], np.float32)
    scene.add_mesh(v, np.array([[0, 1, 2], [0, 2, 3]], np.uint32),
                   ol.Material(base_color=(0.6, 0.5, 0.4), roughness=0.45, metallic=0.0))
    scene.set_environment(ol.EnvironmentLight(color=(0.0, 0.0, 0.0), intensity=0.0))
    scene.add_light(light)
    camera = ol.PerspectiveCamera(position=(0.0, 5.0, -8.0), target=(0.0, 0.0, 0.0), vertical_fov_degrees=40.0)
    return scene, camera


def _floor_points(r, camera, w, h):
    o, d = r.camera_rays(camera, w, h, sample=0, frame_index=0)
    t = -o[:, 1] / d[:, 1]
    p = o + d * t[:, None]
    return p, -d


@pytest.mark.parametrize("kind", ["directional", "point"])
def test_single_analytic_light_on_ggx_matches_the_restated_bsdf(native_library, cuda_device, kind):
    """One light, two bounces, black environment: each pixel is exactly the
    light's direct term f(v, l) * Le * cos (the bounce escapes to black)."""
    if kind == "directional":
        light = ol.DirectionalLight(direction=(-0.3, -1.0, 0.2), color=(1.0, 0.9, 0.8), intensity=3.0)
    else:
        light = ol.PointLight(position=(1.0, 3.0, 0.5), color=(1.0, 0.8, 0.6), intensity=20.0)
    scene, camera = _floor_scene(light)
    w, h = 40, 30
    with CudaWavefrontRenderer(max_bounces=2, samples_per_pixel=1) as r:
        img = r.render_frame(scene, camera, w, h)
        p, view = _floor_points(r, camera, w, h)
    n = np.broadcast_to(np.array([0.0, 1.0, 0.0]), p.shape)
    if kind == "directional":
        expected = pbr.directional_radiance((0.6, 0.5, 0.4), 0.45, 0.0, n, view, light.direction, light.color,
                                            light.intensity)
    else:
        expected = pbr.point_radiance((0.6, 0.5, 0.4), 0.45, 0.0, p, n, view, light.position, light.color,
                                      light.intensity)
    np.testing.assert_allclose(img[..., :3].reshape(-1, 3), expected, rtol=2e-3, atol=1e-6)


def _batches(r, scene, camera, w, h, spp, k, first=0):
    return np.stack([r.render_frame(scene, camera, w, h, samples=spp, frame_index=first + i)[..., :3]
                     for i in range(k)]).astype(np.float64)


def _compare(a, b, rel_bias):
    ma, mb = a.mean(axis=0), b.mean(axis=0)
    ia, ib = a.reshape(len(a), -1, 3).mean(axis=1), b.reshape(len(b), -1, 3).mean(axis=1)
    se = np.sqrt(ia.var(axis=0, ddof=1) / len(ia) + ib.var(axis=0, ddof=1) / len(ib))
    diff = np.abs(ia.mean(axis=0) - ib.mean(axis=0))
    noise = np.mean(a.var(axis=0, ddof=1) / len(a) + b.var(axis=0, ddof=1) / len(b))
    rmse2 = np.mean((ma - mb) ** 2)
    bias = np.sqrt(max(rmse2 - noise, 0.0)) / np.sqrt(np.mean(mb ** 2))
    return diff, se, bias


def test_next_event_estimation_with_mis_is_unbiased(native_library, cuda_device):
    """NEE + power-heuristic MIS and pure BSDF sampling estimate the same
    image (box room, production BSDF)."""
    scene, camera = scenes.box_room()
    w, h = 48, 48
    with CudaWavefrontRenderer(max_bounces=5, russian_roulette_start=0) as r:
        with_nee = _batches(r, scene, camera, w, h, 512, 16)
    with CudaWavefrontRenderer(max_bounces=5, russian_roulette_start=0, nee=False) as r:
        without = _batches(r, scene, camera, w, h, 512, 16, first=100)
    diff, se, bias = _compare(with_nee, without, 0.01)
    assert np.all(diff <= 3.0 * se), f"image means differ by {diff}, 3 SE = {3 * se}"
    assert bias < 0.01, f"noise-corrected relative RMSE {bias:.4f}"


def test_russian_roulette_is_unbiased(native_library, cuda_device):
    scene, camera = scenes.box_room()
    w, h = 48, 48
    with CudaWavefrontRenderer(max_bounces=6, russian_roulette_start=0) as r:
        plain = _batches(r, scene, camera, w, h, 256, 16)
    with CudaWavefrontRenderer(max_bounces=6, russian_roulette_start=2, russian_roulette_min_survival=0.1) as r:
        rr = _batches(r, scene, camera, w, h, 256, 16, first=50)
    diff, se, bias = _compare(plain, rr, 0.01)
    assert np.all(diff <= 3.0 * se), f"image means differ by {diff}, 3 SE = {3 * se}"
    assert bias < 0.01, f"noise-corrected relative RMSE {bias:.4f}"


def test_restir_matches_plain_nee(native_library, cuda_device):
    """ReSTIR DI (initial RIS + spatial reuse, no temporal history) against
    one-sample NEE on an instanced scene with 64 emitters."""
    scene, camera = scenes.instanced_spheres(seed=7, instances=8, segments=32, bands=17, emitters=64, extent=6.0)
    w, h = 64, 48
    with CudaWavefrontRenderer(max_bounces=2, russian_roulette_start=0) as r:
        nee = _batches(r, scene, camera, w, h, 64, 16)
    with CudaWavefrontRenderer(max_bounces=2, russian_roulette_start=0, restir=True, restir_temporal=False) as r:
        restir = _batches(r, scene, camera, w, h, 64, 16, first=40)
    diff, se, bias = _compare(nee, restir, 0.02)
    mean = nee.reshape(len(nee), -1, 3).mean(axis=(0, 1))
    assert np.all(diff <= 3.0 * se + 0.02 * mean), f"image means differ by {diff}, 3 SE = {3 * se}, mean {mean}"
    assert bias < 0.03, f"noise-corrected relative RMSE {bias:.4f}"


def test_restir_lowers_the_error_of_one_sample_frames(native_library, cuda_device):
    """The quality gate of ReSTIR DI (after the reference's error ratio
    against the conventional estimator): with the 64 emitters as the only
    light (black environment, whose BSDF-sampled noise is the same in both
    modes), one-sample frames with 32 resampled candidates and spatial reuse
    are closer to the converged image than one-sample NEE frames on the
    surfaces the emitters light."""
    scene, camera = scenes.instanced_spheres(seed=7, instances=8, segments=32, bands=17, emitters=64, extent=6.0)
    scene.set_environment(ol.EnvironmentLight(color=(0.0, 0.0, 0.0), intensity=0.0))
    w, h = 64, 48
    with CudaWavefrontRenderer(max_bounces=2, russian_roulette_start=0) as r:
        converged = _batches(r, scene, camera, w, h, 256, 8, first=500).mean(axis=0)
        nee = _batches(r, scene, camera, w, h, 1, 16, first=10)
    with CudaWavefrontRenderer(max_bounces=2, russian_roulette_start=0, restir=True, restir_temporal=False,
                               restir_candidates=32, restir_spatial=1) as r:
        restir = _batches(r, scene, camera, w, h, 1, 16, first=10)
    # pixels that see an emitter (or its jittered edge) carry the camera's
    # own sampling noise, the same in both modes: measure the lit surfaces
    lum = converged @ np.array([0.2126, 0.7152, 0.0722])
    lit = (lum > 0.0) & (lum < 10.0 * np.median(lum[lum > 0.0]))
    assert lit.mean() > 0.5
    scale = np.sqrt(np.mean(converged[lit] ** 2))

    def rel_rmse(frames):
        return float(np.mean([np.sqrt(np.mean((f[lit] - converged[lit]) ** 2)) for f in frames]) / scale)

    e_nee, e_restir = rel_rmse(nee), rel_rmse(restir)
    assert e_restir < 0.85 * e_nee, f"ReSTIR error {e_restir:.4f} vs NEE {e_nee:.4f}"


def test_restir_sequences_are_reproducible(native_library, cuda_device):
    scene, camera = scenes.instanced_spheres(seed=7, instances=4, segments=24, bands=13, emitters=32, extent=5.0)
    runs = []
    for _ in range(2):
        with CudaWavefrontRenderer(max_bounces=3, samples_per_pixel=2, restir=True) as r:
            frames = [r.render_frame(scene, camera, 40, 30, frame_index=k) for k in range(3)]
            used = r.last_timings["restir_history_used"]
        runs.append(frames)
        assert used  # frames 1 and 2 reuse the previous frame's reservoirs
    for a, b in zip(*runs):
        assert a.tobytes() == b.tobytes()


def test_render_products_follow_the_primary_hits(native_library, cuda_device):
    scene, camera = scenes.box_room()
    w, h = 48, 40
    with CudaWavefrontRenderer(mode="reference_compatible", max_bounces=2, samples_per_pixel=2) as r:
        prods = r.render_products(scene, camera, w, h, outputs=("color", "depth", "normal", "instance_id",
                                                                 "material_id"))
        o, d = r.camera_rays(camera, w, h, sample=0, frame_index=0)
        inst, prim, t, _ = r.trace_closest(scene, o, d, t_min=1e-4)
    assert prods["color"].shape == (h, w, 4) and prods["depth"].shape == (h, w)
    assert prods["normal"].shape == (h, w, 3) and prods["instance_id"].dtype == np.uint32
    np.testing.assert_array_equal(prods["instance_id"].reshape(-1), inst)
    hit = prim >= 0
    np.testing.assert_allclose(prods["depth"].reshape(-1)[hit], t[hit], rtol=1e-6)
    assert np.all(np.isinf(prods["depth"].reshape(-1)[~hit]))
    mats = {scene.material_id(m.material) for m in scene.meshes}
    assert set(np.unique(prods["material_id"].reshape(-1)[hit]).tolist()) <= mats


@pytest.mark.parametrize("restir", [False, True])
def test_variance_product_is_the_sample_variance_of_the_samples(native_library, cuda_device, restir):
    from ordinarylight_b200.renderers.cuda import RenderRequest

    scene, camera = scenes.instanced_spheres(seed=7, instances=6, segments=24, bands=13, emitters=32)
    w, h, spp = 40, 32, 6
    with CudaWavefrontRenderer(max_bounces=4, restir=restir) as r:
        prods = r.render_products(scene, camera, w, h, outputs=("color", "variance"), samples=spp, frame_index=3)
        per_sample = r.render_batch([RenderRequest(scene, camera, w, h, samples=1, frame_index=3, first_sample=s)
                                     for s in range(spp)])
        one = r.render_products(scene, camera, w, h, outputs="variance", samples=1, frame_index=4)["variance"]
    var = prods["variance"]
    assert var.shape == (h, w) and var.dtype == np.float32
    assert var.tobytes() == products.sample_variance([img[..., :3] for img in per_sample]).tobytes()
    assert np.count_nonzero(var) > var.size // 10
    assert not one.any()


def _glass_cube(size, angles, center):
    """Cube with one vertex set per face and face normals, so that shading
    normals equal geometric ones."""
    ax, ay = angles
    rx = np.array([[1, 0, 0], [0, np.cos(ax), -np.sin(ax)], [0, np.sin(ax), np.cos(ax)]])
    ry = np.array([[np.cos(ay), 0, np.sin(ay)], [0, 1, 0], [-np.sin(ay), 0, np.cos(ay)]])
    rot = ry @ rx
    h = size / 2.0
    faces = []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            n = np.zeros(3)
            n[axis] = sign
            u = np.zeros(3)
            u[(axis + 1) % 3] = h
            w = np.cross(n, u)
            c = n * h
            quad = [c - u - w, c + u - w, c + u + w, c - u + w]
            faces.append((quad, n))
    verts, norms, idx = [], [], []
    for quad, n in faces:
        b = len(verts)
        verts += [rot @ q + center for q in quad]
        norms += [rot @ n] * 4
        idx += [(b, b + 1, b + 2), (b, b + 2, b + 3)]
    return np.array(verts, np.float32), np.array(idx, np.uint32), np.array(norms, np.float32)


def test_dielectric_interfaces_match_the_restated_refraction(native_library, cuda_device):
    """Nested glass cubes (IOR 1.5 around IOR 1.25) under an equirect
    environment: each pixel's path is deterministic (refraction, total
    internal reflection, the medium stack), so every robust pixel must equal
    the oracle's deterministic trace of the same camera ray."""
    from oracle import dielectric

    rng = np.random.default_rng(12)
    scene = ol.Scene()
    outer = dict(base_color=(0.6, 0.8, 1.0), transmission=0.9, ior=1.5, roughness=0.0)
    inner = dict(base_color=(1.0, 0.7, 0.5), transmission=1.0, ior=1.25, roughness=0.0)
    tri_props = []
    for size, angles, props in ((3.0, (0.5, 0.7), outer), (1.3, (-0.3, 0.9), inner)):
        v, i, n = _glass_cube(size, angles, np.zeros(3))
        scene.add_mesh(v, i, ol.Material(**props), normals=n)
        tri_props.append((v[i], props))
    env = rng.uniform(0.05, 2.0, (16, 32, 3)).astype(np.float32)
    scene.set_environment(ol.EnvironmentLight(image=env))
    camera = ol.PerspectiveCamera(position=(0.3, 0.8, -7.0), target=(0.0, 0.0, 0.0), vertical_fov_degrees=35.0)
    w, h, bounces = 96, 80, 16
    with CudaWavefrontRenderer(max_bounces=bounces, samples_per_pixel=1, russian_roulette_start=0) as r:
        img = r.render_frame(scene, camera, w, h, frame_index=5)
        o, d = r.camera_rays(camera, w, h, sample=0, frame_index=5)
    tris = np.concatenate([t for t, _ in tri_props])
    transmission = np.concatenate([np.full(len(t), p["transmission"]) for t, p in tri_props])
    ior = np.concatenate([np.full(len(t), p["ior"]) for t, p in tri_props])
    base = np.concatenate([np.tile(np.asarray(p["base_color"]), (len(t), 1)) for t, p in tri_props])
    expected, robust = dielectric.trace(np.asarray(o), np.asarray(d), tris, transmission, ior, base, env,
                                        max_bounces=bounces)
    got = img[..., :3].reshape(-1, 3)
    hit_glass = np.any(np.abs(expected - dielectric.trace(np.asarray(o), np.asarray(d), tris[:0], transmission[:0],
                                                          ior[:0], base[:0], env, max_bounces=1)[0]) > 0, axis=1)
    assert robust.mean() > 0.9 and (robust & hit_glass).sum() > w * h // 5
    np.testing.assert_allclose(got[robust], expected[robust], rtol=1e-4, atol=1e-6)


def test_deeply_nested_dielectrics_use_the_full_medium_stack(native_library, cuda_device):
    """Twelve nested glass cubes: rays through the centre enter twelve media
    (stack depth 13 of the reference's 16), so every interface's IOR ratio
    comes from the stack; robust pixels must equal the oracle's trace (all
    but a handful that float32 rounding sends to another texel)."""
    from oracle import dielectric

    rng = np.random.default_rng(31)
    scene = ol.Scene()
    tri_props = []
    angles = (0.45, 0.6)          # one orientation: the cubes nest without touching
    for k in range(12):
        size = 3.0 - 0.2 * k
        props = dict(base_color=(1.0, 1.0, 1.0), transmission=1.0, ior=1.6 if k % 2 == 0 else 1.3, roughness=0.0)
        v, i, n = _glass_cube(size, angles, np.zeros(3))
        scene.add_mesh(v, i, ol.Material(**props), normals=n)
        tri_props.append((v[i], props))
    env = rng.uniform(0.05, 2.0, (16, 32, 3)).astype(np.float32)
    scene.set_environment(ol.EnvironmentLight(image=env))
    camera = ol.PerspectiveCamera(position=(0.2, 0.3, -6.0), target=(0.0, 0.0, 0.0), vertical_fov_degrees=22.0)
    w, h, bounces = 48, 40, 40
    with CudaWavefrontRenderer(max_bounces=bounces, samples_per_pixel=1, russian_roulette_start=0) as r:
        img = r.render_frame(scene, camera, w, h, frame_index=1)
        o, d = r.camera_rays(camera, w, h, sample=0, frame_index=1)
    tris = np.concatenate([t for t, _ in tri_props])
    transmission = np.concatenate([np.full(len(t), p["transmission"]) for t, p in tri_props])
    ior = np.concatenate([np.full(len(t), p["ior"]) for t, p in tri_props])
    base = np.concatenate([np.tile(np.asarray(p["base_color"]), (len(t), 1)) for t, p in tri_props])
    expected, robust = dielectric.trace(np.asarray(o), np.asarray(d), tris, transmission, ior, base, env,
                                        max_bounces=bounces, max_depth=16)
    assert robust.mean() > 0.4
    # after ~25 refractions float32 and float64 directions can part at an
    # environment texel border the oracle did not flag: allow 0.5 % of pixels
    got = img[..., :3].reshape(-1, 3)[robust]
    close = np.all(np.abs(got - expected[robust]) <= 1e-6 + 2e-4 * np.abs(expected[robust]), axis=1)
    assert close.mean() >= 0.995
