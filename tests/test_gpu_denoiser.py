"""Denoiser input signals (capture_denoiser_raw / capture_denoiser_signals,
ordinarylight/targets/vulkan/api.py:1453-1660) against the reference's
definitions restated on the captured products: the diffuse/specular
partition by the primary material's specular-lobe probability, the
next-vertex hit distance, view depth, normals and roughness, and the
canonical motion (previous-minus-current from the pixel centre)."""

from __future__ import annotations

import numpy as np
import pytest

import ordinarylight_b200 as ol
from oracle import products
from ordinarylight_b200 import CudaWavefrontRenderer

pytestmark = pytest.mark.gpu

FLOOR = dict(base_color=(0.8, 0.2, 0.1), metallic=0.7, roughness=0.35)
WALL = dict(base_color=(0.5, 0.5, 0.5), metallic=0.0, roughness=0.9)


def _scene():
    scene = ol.Scene()
    quad = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    scene.add_mesh(np.array([[-8, 0, -8], [-8, 0, 8], [8, 0, 8], [8, 0, -8]], np.float32), quad, ol.Material(**FLOOR))
    scene.add_mesh(np.array([[-8, 0, 6], [-8, 8, 6], [8, 8, 6], [8, 0, 6]], np.float32), quad, ol.Material(**WALL))
    scene.add_mesh(np.array([[-1, 5, 2], [1, 5, 2], [1, 5, 4], [-1, 5, 4]], np.float32), quad,
                   ol.Material(base_color=(0, 0, 0), emission=(20.0, 18.0, 15.0), emission_two_sided=True))
    camera = ol.PerspectiveCamera(position=(0.5, 3.0, -6.0), target=(0.0, 1.0, 2.0), vertical_fov_degrees=50.0)
    return scene, camera


def _spec_probability(m):
    f0 = 0.04 + (np.asarray(m["base_color"]) - 0.04) * m["metallic"]
    return float(np.clip(f0.max(), 0.1, 0.9))


def test_raw_capture_partitions_radiance_and_records_the_next_vertex(native_library, cuda_device):
    scene, camera = _scene()
    w, h = 64, 48
    with CudaWavefrontRenderer(max_bounces=4, denoiser_signal_capture=True) as r:
        raw = r.capture_denoiser_raw(scene, camera, w, h, frame_index=3)
        plain = r.render_frame(scene, camera, w, h, samples=1, frame_index=3)
    ps = raw["path_state"]
    diffuse, specular = ps["diffuse_radiance_hit_distance"], ps["specular_radiance_hit_distance"]
    assert raw["radiance"].tobytes() == plain.tobytes()        # the capture is the one-sample frame
    np.testing.assert_allclose(diffuse[..., :3] + specular[..., :3], np.maximum(plain[..., :3], 0.0), rtol=1e-6)
    prim = raw["primitive_id"]
    expected = np.zeros((h, w), np.float32)
    expected[(prim == 0) | (prim == 1)] = _spec_probability(FLOOR)
    expected[(prim == 2) | (prim == 3)] = _spec_probability(WALL)
    expected[(prim == 4) | (prim == 5)] = 0.1                   # the emitter: black base, not metallic
    np.testing.assert_allclose(ps["specular_probability"], expected, rtol=1e-6, atol=1e-7)
    # the next vertex lies on one of the scene's planes, at the recorded distance
    sec = ps["secondary_position"]
    valid = sec[..., 3] > 0.5
    assert valid.mean() > 0.2            # the scene is open: many bounces leave it
    p = sec[valid, :3]
    on_plane = (np.abs(p[:, 1]) < 1e-3) | (np.abs(p[:, 2] - 6.0) < 1e-3) | (np.abs(p[:, 1] - 5.0) < 1e-3)
    assert on_plane.all()
    dist = np.linalg.norm(p - raw["primary_position"][valid], axis=-1)
    np.testing.assert_allclose(diffuse[valid, 3], dist, rtol=1e-6)
    assert (diffuse[~valid, 3] == 0).all() and (specular[..., 3] == diffuse[..., 3]).all()


def test_signals_view_depth_normals_and_canonical_motion(native_library, cuda_device):
    from ordinarylight_b200.denoising import camera_matrix

    scene, camera = _scene()
    w, h = 64, 48
    moved = ol.PerspectiveCamera(position=(0.9, 3.2, -5.7), target=(0.1, 1.0, 2.2), vertical_fov_degrees=50.0)
    with CudaWavefrontRenderer(max_bounces=3, denoiser_signal_capture=True) as r:
        first = r.capture_denoiser_signals(scene, camera, w, h, frame_index=0)
        before = products.capture_state(scene, camera, (w, h))
        second = r.capture_denoiser_signals(scene, moved, w, h, frame_index=1)
        prim = r.primitive_ids(w, h)
        pos, bary = r.hit_geometry(w, h)
    assert first.frame.camera_cut and not first.motion.any()
    assert not second.frame.camera_cut and second.frame.frame_index == 1
    np.testing.assert_allclose(second.frame.world_to_clip, camera_matrix(moved, w, h))
    np.testing.assert_allclose(second.frame.previous_world_to_clip, camera_matrix(camera, w, h))
    fg = prim != 0xFFFFFFFF
    origin = np.asarray(moved.position, np.float64)
    fwd = np.asarray(moved.target, np.float64) - origin
    fwd /= np.linalg.norm(fwd)
    np.testing.assert_allclose(second.view_z[fg], (pos[fg] - origin) @ fwd, rtol=1e-5)
    assert (second.view_z[~fg] == 0).all()
    np.testing.assert_allclose(np.linalg.norm(second.normal_roughness[fg, :3], axis=-1), 1.0, atol=1e-5)
    rough = second.normal_roughness[..., 3]
    assert np.allclose(rough[(prim == 0) | (prim == 1)], FLOOR["roughness"])
    assert np.allclose(rough[(prim == 2) | (prim == 3)], WALL["roughness"])
    # canonical motion: projected hit point minus pixel centre minus the
    # general (current-minus-previous) motion product
    general = products.motion_product(before, scene, moved, w, h, prim, pos, bary)
    proj, ok = products.project_positions(pos.reshape(-1, 3), moved, w, h)
    yy, xx = np.indices((h, w))
    expected = proj.reshape(h, w, 2) - (np.stack((xx, yy), axis=-1) + 0.5) - general
    expected[~(fg & ok.reshape(h, w))] = 0.0
    np.testing.assert_allclose(second.motion, expected, atol=2e-3)
    assert np.abs(second.motion[fg]).max() > 0.1
