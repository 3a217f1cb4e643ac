"""GPU parity of the core stages against the oracle and the reference's
golden fixtures: LBVH keys and order, camera rays, primary-hit IDs."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import lbvh, reference_path_tracer as ref, sampling
from ordinarylight_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def renderer(native_library, cuda_device):
    from ordinarylight_b200 import CudaWavefrontRenderer

    r = CudaWavefrontRenderer(mode="reference_compatible", max_bounces=4, samples_per_pixel=1)
    yield r
    r.close()


def _device_codes(renderer, tris):
    import torch

    t = torch.as_tensor(np.ascontiguousarray(tris, np.float32).reshape(-1, 9), device="cuda")
    codes = torch.empty(len(tris), dtype=torch.int32, device="cuda")
    lib = renderer._lib
    from ordinarylight_b200 import _native

    _native.check(lib, renderer._ctx, lib.olc_morton_codes(renderer._ctx, len(tris), _native.ptr(t),
                                                           _native.ptr(codes)))
    return codes.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n", [1, 2, 37, 2048, 2049, 100_000, 1_000_003])
def test_morton_codes_bit_exact(renderer, n):
    rng = np.random.default_rng(n)
    tris = (rng.normal(size=(n, 3, 3)) * rng.uniform(0.1, 100.0)).astype(np.float32)
    np.testing.assert_array_equal(_device_codes(renderer, tris), lbvh.morton_codes(tris))


@pytest.mark.parametrize("n,bits", [(1, 30), (5, 30), (2047, 30), (2048, 30), (4097, 8), (300_001, 30),
                                    (2_000_000, 30), (65_537, 32)])
def test_radix_sort_equals_stable_host_sort(renderer, n, bits):
    import torch
    from ordinarylight_b200 import _native

    rng = np.random.default_rng(7 + n)
    # keys drawn from a small pool so equal keys are common and stability matters
    pool = rng.integers(0, 1 << bits, size=max(2, n // 10), dtype=np.uint64)
    keys = rng.choice(pool, size=n).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    k = torch.as_tensor(keys.view(np.int32).copy(), device="cuda")
    v = torch.as_tensor(vals.view(np.int32).copy(), device="cuda")
    lib = renderer._lib
    _native.check(lib, renderer._ctx, lib.olc_radix_sort_pairs(renderer._ctx, n, bits, _native.ptr(k),
                                                               _native.ptr(v)))
    order = np.argsort(keys & np.uint32((1 << bits) - 1 if bits < 32 else 0xFFFFFFFF), kind="stable")
    np.testing.assert_array_equal(v.cpu().numpy().view(np.uint32), order.astype(np.uint32))
    np.testing.assert_array_equal(k.cpu().numpy().view(np.uint32), keys[order])


def test_bvh_structure_is_valid(renderer):
    for scene in (scenes.box_room()[0],
                  scenes.instanced_spheres(seed=5, instances=3, segments=32, bands=17, emitters=8)[0]):
        assert renderer.validate_bvh(scene) == 0


def _classify(gpu_prim, gpu_t, cpu_prim, cpu_t):
    """Mismatches must be ties: both hit, |t_gpu - t_cpu| within 1 ulp."""
    mismatch = gpu_prim != cpu_prim
    ties = mismatch & (gpu_prim >= 0) & (cpu_prim >= 0)
    ulp = np.spacing(np.maximum(np.abs(cpu_t[ties]), np.abs(gpu_t[ties])).astype(np.float32))
    tie_ok = np.abs(gpu_t[ties] - cpu_t[ties]) <= ulp
    return int(mismatch.sum()), int(ties.sum()), int(tie_ok.sum())


def test_primary_hit_ids_match_reference_on_identical_rays(renderer, golden):
    data = golden("config1_primary.npz")
    scene, camera = scenes.box_room()
    o, d = ref.camera_rays(camera, 256, 256, np.random.default_rng(1))
    o32, d32 = o.astype(np.float32), d.astype(np.float32)
    inst, prim, t, _bary = renderer.trace_closest(scene, o32, d32, t_min=1e-4)
    cpu_prim = data["triangle"].astype(np.int32)
    mismatches, ties, tie_ok = _classify(prim, t, cpu_prim, data["t"])
    assert mismatches == tie_ok, f"{mismatches} mismatches, {ties} both-hit, {tie_ok} t-ties within 1 ulp"
    hit = cpu_prim >= 0
    ids = scene.triangle_instance_ids()
    np.testing.assert_array_equal(inst[hit & (prim == cpu_prim)], ids[cpu_prim[hit & (prim == cpu_prim)]])
    np.testing.assert_allclose(t[hit], data["t"][hit], rtol=2e-5)


def test_primary_hit_ids_instanced_scene(renderer, golden):
    data = golden("spheres_small.npz")
    scene, _camera = scenes.instanced_spheres(seed=5, instances=2, segments=16, bands=9, emitters=4, extent=3.0)
    np.testing.assert_array_equal(scene.triangles()[0], data["triangles"])
    inst, prim, t, _ = renderer.trace_closest(scene, data["origins"], data["directions"], t_min=1e-4)
    mismatches, _ties, tie_ok = _classify(prim, t, data["triangle"], data["t"])
    assert mismatches == tie_ok
    assert int((prim >= 0).sum()) > 100


def test_closest_hit_matches_oracle_on_random_rays(renderer):
    scene, _ = scenes.instanced_spheres(seed=11, instances=6, segments=24, bands=13, emitters=16, extent=4.0)
    tris = scene.triangles()[0]
    rng = np.random.default_rng(5)
    n = 3000
    o = rng.uniform(-8, 8, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    _inst, prim, t, _ = renderer.trace_closest(scene, o, d, t_min=1e-4)
    cpu_t, cpu_prim = ref.intersect(o, d, tris)
    mismatches, _ties, tie_ok = _classify(prim, t, cpu_prim, cpu_t)
    assert mismatches == tie_ok


def test_occlusion_agrees_with_closest_hit(renderer):
    scene, _ = scenes.instanced_spheres(seed=12, instances=5, segments=24, bands=13, emitters=0, extent=4.0)
    rng = np.random.default_rng(6)
    n = 4000
    o = rng.uniform(-8, 8, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    _i, prim, t, _ = renderer.trace_closest(scene, o, d, t_min=1e-3)
    tmax = np.full(n, 5.0, np.float32)
    occ = renderer.trace_occluded(scene, o, d, tmax, t_min=1e-3)
    expect = (prim >= 0) & (t <= 5.0)
    assert np.array_equal(occ, expect)


def test_camera_rays_follow_the_reference_camera_model(renderer):
    _scene, camera = scenes.box_room()
    w, h = 64, 48
    o, d = renderer.camera_rays(camera, w, h, sample=3, frame_index=5)
    jx, jy = sampling.camera_jitter(np.arange(w * h, dtype=np.uint32), 3, 1 + 5)
    # reference camera model with the device jitter (float64 like the reference)
    pos, fwd, right, up = (np.asarray(v, np.float64) for v in _basis(camera))
    ys, xs = np.divmod(np.arange(w * h), w)
    ndc_x = (xs + jx.astype(np.float64)) / w * 2.0 - 1.0
    ndc_y = 1.0 - (ys + jy.astype(np.float64)) / h * 2.0
    half = math.tan(math.radians(camera.vertical_fov_degrees) / 2.0)
    dirs = fwd + ndc_x[:, None] * (w / h * half) * right + ndc_y[:, None] * half * up
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    np.testing.assert_allclose(d, dirs, atol=3e-6)
    np.testing.assert_array_equal(o, np.repeat(pos[None].astype(np.float32), w * h, axis=0))


def _expected_rays(camera, w, h, jx, jy):
    """The reference camera model (path_tracer.py:110-151) in float64 with
    the device's jitter: orthographic origins on the image plane along the
    forward direction; panoramic yaw and pitch proportional to NDC."""
    import ordinarylight_b200 as ol

    pos, fwd, right, up = (np.asarray(v, np.float64) for v in _basis(camera))
    ys, xs = np.divmod(np.arange(w * h), w)
    ndc_x = (xs + jx.astype(np.float64)) / w * 2.0 - 1.0
    ndc_y = 1.0 - (ys + jy.astype(np.float64)) / h * 2.0
    if isinstance(camera, ol.OrthographicCamera):
        half = camera.vertical_size * 0.5
        origins = pos + ndc_x[:, None] * (w / h * half) * right + ndc_y[:, None] * half * up
        dirs = np.repeat((fwd / np.linalg.norm(fwd))[None], w * h, axis=0)
    else:
        yaw = ndc_x * math.radians(camera.horizontal_fov_degrees) * 0.5
        pitch = ndc_y * math.radians(camera.vertical_fov_degrees) * 0.5
        dirs = (np.cos(pitch)[:, None] * np.cos(yaw)[:, None] * fwd + np.cos(pitch)[:, None] * np.sin(yaw)[:, None]
                * right + np.sin(pitch)[:, None] * up)
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        origins = np.repeat(pos[None], w * h, axis=0)
    return origins, dirs


@pytest.mark.parametrize("kind", ["orthographic", "panoramic"])
def test_orthographic_and_panoramic_rays_follow_the_reference_camera_model(renderer, kind):
    import ordinarylight_b200 as ol

    if kind == "orthographic":
        camera = ol.OrthographicCamera(position=(0.3, 1.2, -4.0), target=(0.0, 0.5, 0.0), vertical_size=3.0)
    else:
        camera = ol.PanoramicCamera(position=(0.3, 1.2, -4.0), target=(0.0, 0.5, 0.0),
                                    horizontal_fov_degrees=300.0, vertical_fov_degrees=150.0)
    w, h = 64, 48
    o, d = renderer.camera_rays(camera, w, h, sample=3, frame_index=5)
    jx, jy = sampling.camera_jitter(np.arange(w * h, dtype=np.uint32), 3, 1 + 5)
    origins, dirs = _expected_rays(camera, w, h, jx, jy)
    # float32 device arithmetic (sinf/cosf, products of unit vectors)
    np.testing.assert_allclose(d, dirs, atol=1e-5)
    np.testing.assert_allclose(o, origins, atol=2e-5)


def _basis(camera):
    from ordinarylight_b200.packing import camera_basis

    return camera_basis(camera)


def test_flattened_small_instances_hit_the_same_primitives(native_library, cuda_device, golden):
    """Baking small instances into one world-space mesh changes no primary-hit
    ID (beyond t-ties) and reports the original instance IDs."""
    from ordinarylight_b200 import CudaWavefrontRenderer

    data = golden("spheres_small.npz")
    scene, _camera = scenes.instanced_spheres(seed=5, instances=2, segments=16, bands=9, emitters=4, extent=3.0)
    results = []
    for flatten in (True, False):
        with CudaWavefrontRenderer(mode="reference_compatible", flatten_instances=flatten) as r:
            results.append(r.trace_closest(scene, data["origins"], data["directions"], t_min=1e-4))
            assert r.validate_bvh(scene) == 0
    for inst, prim, t, _ in results:
        mismatches, _ties, tie_ok = _classify(prim, t, data["triangle"], data["t"])
        assert mismatches == tie_ok
        ids = scene.triangle_instance_ids()
        ok = prim >= 0
        np.testing.assert_array_equal(inst[ok], ids[prim[ok]])


@pytest.mark.parametrize("grid", [256, 300])
def test_both_hierarchy_builders_give_valid_trees_and_the_oracles_hits(renderer, grid):
    """A heightfield of 2 (grid - 1)^2 triangles: 130,050 (binned SAH on the
    host, up to 131,072 primitives) and 178,802 (the device's Morton-order
    build).  Either tree validates and gives the closest hits of the
    oracle's own hierarchy (oracle/transport.c), up to exact ties."""
    import ordinarylight_b200 as ol
    from oracle import production

    heights = scenes.fbm_heightfield(grid, seed=9, octaves=4, amplitude=6.0)
    v, i = scenes.grid_mesh(heights, 0.25)
    scene = ol.Scene()
    scene.add_mesh(v, i, ol.Material(base_color=(0.5, 0.5, 0.5)))
    assert renderer.validate_bvh(scene) == 0
    rng = np.random.default_rng(grid)
    n = 20000
    o = np.column_stack([rng.uniform(-30, 30, n), np.full(n, 20.0), rng.uniform(-30, 30, n)]).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d[:, 1] = -np.abs(d[:, 1]) - 0.2
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    _inst, prim, t, _ = renderer.trace_closest(scene, o, d, t_min=1e-4)
    cpu_prim, cpu_t = production.trace(scene, o, d, t_min=1e-4)
    assert int((cpu_prim >= 0).sum()) > n // 2
    mismatches, _ties, tie_ok = _classify(prim, t, cpu_prim, cpu_t.astype(np.float32))
    assert mismatches == tie_ok
    hit = cpu_prim >= 0
    np.testing.assert_allclose(t[hit], cpu_t[hit], rtol=1e-4)
