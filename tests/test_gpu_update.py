"""In-place scene updates (refit for deformation, TLAS rebuild for moved
instances) against uploading the changed scene from scratch.

A transform-only update rebuilds the TLAS from the same boxes a fresh upload
uses, so its frames equal a fresh renderer's bit for bit.  A refit keeps the
BVH topology of the first build, so after a deformation the hierarchy
differs from a rebuild's; closest hits are then the same up to exact ties,
and the refit hierarchy must still be valid (every triangle reachable once,
every child box inside its parent).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import ordinarylight_b200 as ol
from ordinarylight_b200 import CudaWavefrontRenderer, _native, scenes
from ordinarylight_b200.packing import pack_scene
from ordinarylight_b200.renderers.cuda import RenderRequest

pytestmark = pytest.mark.gpu

W, H, SPP = 48, 40, 3


def _animated_scene(seed=3):
    rng = np.random.default_rng(seed)
    scene = ol.Scene()
    v, i, n = scenes.uv_sphere(24, 13)
    blob = scene.create_mesh(v, i, ol.Material(), normals=n, name="blob", deformable=True)
    xfs, mats = [], []
    for _ in range(5):
        xf = np.eye(4, dtype=np.float32)
        xf[:3, :3] *= rng.uniform(0.6, 1.4)
        xf[:3, 3] = rng.uniform(-3.0, 3.0, 3)
        xfs.append(ol.Transform(xf))
        mats.append(ol.Material(base_color=tuple(float(c) for c in rng.uniform(0.2, 0.9, 3)),
                                roughness=float(rng.uniform(0.1, 0.9)), metallic=float(rng.random() < 0.3)))
    inst = scene.add_instances(blob, xfs, materials=mats)
    gv = np.array([[-12, -4, -12], [-12, -4, 12], [12, -4, 12], [12, -4, -12]], np.float32)
    scene.add_mesh(gv, np.array([[0, 1, 2], [0, 2, 3]], np.uint32),
                   ol.Material(base_color=(0.5, 0.5, 0.5), roughness=0.7))
    tri = scene.create_mesh(np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1]], np.float32), np.array([[0, 2, 1]], np.uint32),
                            ol.Material(), name="emitter")
    exf, emat = [], []
    for _ in range(6):
        xf = np.eye(4, dtype=np.float32)
        xf[:3, 3] = rng.uniform(-4.0, 4.0, 3) + np.array([0.0, 5.0, 0.0])
        exf.append(ol.Transform(xf))
        emat.append(ol.Material(base_color=(0, 0, 0), emission=tuple(float(c) for c in rng.uniform(5, 30, 3))))
    lights = scene.add_instances(tri, exf, materials=emat)
    camera = ol.PerspectiveCamera(position=(0.0, 3.0, -12.0), target=(0.0, 0.0, 0.0), vertical_fov_degrees=45.0)
    return scene, camera, blob, inst, lights


def _moved(instances, rng):
    out = []
    for inst in instances:
        m = np.array(inst.transform.matrix, np.float32)
        m[:3, 3] += rng.uniform(-0.7, 0.7, 3)
        out.append(ol.Transform(m))
    return out


def _deformed(vertices, phase):
    v = np.array(vertices, np.float64)
    r = 1.0 + 0.15 * np.sin(3.0 * v[:, 0] + phase) * np.cos(2.0 * v[:, 1])
    return (v * r[:, None]).astype(np.float32)


def _fresh(scene, camera, frame_index, **cfg):
    with CudaWavefrontRenderer(max_bounces=4, **cfg) as r:
        return r.render_frame(scene, camera, W, H, samples=SPP, frame_index=frame_index)


@pytest.mark.parametrize("restir", [False, True])
def test_moved_instances_render_like_a_fresh_upload(native_library, cuda_device, restir):
    scene, camera, _blob, inst, lights = _animated_scene()
    rng = np.random.default_rng(11)
    with CudaWavefrontRenderer(max_bounces=4, restir=restir) as r:
        r.render_frame(scene, camera, W, H, samples=SPP, frame_index=0)
        scene.update_instance_transforms(inst[:3] + lights[:2], _moved(inst[:3] + lights[:2], rng))
        img = r.render_frame(scene, camera, W, H, samples=SPP, frame_index=1)
        assert r.last_update == {"refitted_blas": 0, "meshes": 3}
        assert r.validate_bvh(scene) == 0
    assert img.tobytes() == _fresh(scene, camera, 1, restir=restir).tobytes()


def test_refit_of_unchanged_geometry_reproduces_the_frame(native_library, cuda_device):
    scene, camera, *_ = _animated_scene()
    with CudaWavefrontRenderer(max_bounces=4) as r:
        before = r.render_frame(scene, camera, W, H, samples=SPP, frame_index=2)
        packed = pack_scene(scene)      # owns the arrays the descriptor points to
        desc = packed.descriptor()
        applied, refitted = ctypes.c_int32(), ctypes.c_uint32()
        _native.check(r._lib, r._ctx, r._lib.olc_update_scene(r._ctx, _native.DEFAULT_SCENE, ctypes.byref(desc), None,
                                                             ctypes.byref(applied), ctypes.byref(refitted)))
        assert applied.value == 1 and refitted.value >= 1
        after = r.render_frame(scene, camera, W, H, samples=SPP, frame_index=2)
    assert after.tobytes() == before.tobytes()


def test_deformation_refits_and_hits_like_a_rebuild(native_library, cuda_device):
    scene, camera, blob, _inst, _lights = _animated_scene()
    base = np.array(blob.vertices)
    with CudaWavefrontRenderer(max_bounces=4) as r, CudaWavefrontRenderer(max_bounces=4) as fresh:
        r.render_frame(scene, camera, W, H, samples=SPP, frame_index=0)
        for step in range(3):
            scene.update_mesh_resource(blob, vertices=_deformed(base, 0.9 * (step + 1)))
            img = r.render_frame(scene, camera, W, H, samples=SPP, frame_index=step + 1)
            assert r.last_update is not None and r.last_update["refitted_blas"] == 1
            assert r.validate_bvh(scene) == 0
            o, d = r.camera_rays(camera, 160, 120, sample=0, frame_index=0)
            inst_a, prim_a, t_a, _ = r.trace_closest(scene, o, d)
            inst_b, prim_b, t_b, _ = fresh.trace_closest(scene, o, d)
            same = prim_a == prim_b
            assert same.mean() > 0.999
            np.testing.assert_array_equal(t_a[same], t_b[same])
            ref = fresh.render_frame(scene, camera, W, H, samples=SPP, frame_index=step + 1)
            assert (img == ref).all(axis=-1).mean() > 0.99


def test_rigid_mesh_with_new_vertices_is_uploaded_again(native_library, cuda_device):
    scene, camera = scenes.box_room()
    mesh = scene.meshes[0]
    with CudaWavefrontRenderer(max_bounces=3) as r:
        r.render_frame(scene, camera, W, H, samples=SPP, frame_index=0)
        scene.update_mesh_resource(mesh.resource, vertices=np.asarray(mesh.vertices) * 1.01)
        img = r.render_frame(scene, camera, W, H, samples=SPP, frame_index=1)
        assert r.last_update is None
    with CudaWavefrontRenderer(max_bounces=3) as f:
        assert img.tobytes() == f.render_frame(scene, camera, W, H, samples=SPP, frame_index=1).tobytes()


def test_pool_scene_updates_in_place(native_library, cuda_device):
    scene, camera, blob, inst, _lights = _animated_scene(seed=5)
    rng = np.random.default_rng(2)
    req = RenderRequest(scene, camera, W, H, samples=SPP, frame_index=4, max_bounces=4)
    with CudaWavefrontRenderer(max_bounces=4) as r:
        h0 = r.resident_scene(scene)
        r.render_batch([req])
        scene.update_instance_transforms(inst[1:4], _moved(inst[1:4], rng))
        h1 = r.resident_scene(scene)
        assert h1 == h0 and r.last_update is not None
        moved = r.render_batch([req])[0]
        assert len(r.resident_scenes()) == 1
    with CudaWavefrontRenderer(max_bounces=4) as f:
        assert moved.tobytes() == f.render_batch([req])[0].tobytes()


def test_motion_product_matches_the_reference_arithmetic(native_library, cuda_device):
    from oracle import products

    scene, camera, blob, inst, lights = _animated_scene(seed=8)
    rng = np.random.default_rng(4)
    w, h = 64, 48
    with CudaWavefrontRenderer(max_bounces=2) as r:
        first = r.render_products(scene, camera, w, h, outputs=("color", "motion"), samples=1, frame_index=0)
        assert not first["motion"].any()          # no history yet
        before = products.capture_state(scene, camera, (w, h))
        scene.update_instance_transforms(inst[:4], _moved(inst[:4], rng))
        scene.update_mesh_resource(blob, vertices=_deformed(np.array(blob.vertices), 0.4))
        moved_camera = ol.PerspectiveCamera(position=(0.4, 3.2, -11.5), target=(0.1, 0.0, 0.2),
                                            vertical_fov_degrees=45.0)
        out = r.render_products(scene, moved_camera, w, h, outputs=("motion", "depth"), samples=1, frame_index=1)
        prim = r.primitive_ids(w, h)
        pos, bary = r.hit_geometry(w, h)
        expected = products.motion_product(before, scene, moved_camera, w, h, prim, pos, bary)
        assert out["motion"].shape == (h, w, 2) and out["motion"].dtype == np.float32
        np.testing.assert_allclose(out["motion"], expected, atol=2e-3, rtol=0)
        assert np.count_nonzero(np.abs(expected).max(axis=-1) > 0.05) > w * h // 10
        hit = prim != 0xFFFFFFFF
        np.testing.assert_allclose(np.linalg.norm(pos[hit] - np.array(moved_camera.position, np.float32), axis=-1),
                                   out["depth"][hit] * np.linalg.norm(
                                       np.asarray(r.camera_rays(moved_camera, w, h, sample=0, frame_index=1)[1])
                                       .reshape(h, w, 3)[hit], axis=-1), rtol=1e-4)
        # a reset forgets the history
        r.reset_output_history()
        again = r.render_products(scene, moved_camera, w, h, outputs="motion", samples=1, frame_index=2)
        assert not again["motion"].any()
