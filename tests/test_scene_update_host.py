"""Host rules of in-place scene updates (no GPU): which edits refit, which
rewrite records only, and which need a new upload, following the
reference's _try_update_window_scene (targets/vulkan/core.py:4696-4760)."""

from __future__ import annotations

import numpy as np

import ordinarylight_b200 as ol
from ordinarylight_b200 import scenes
from ordinarylight_b200.packing import pack_scene, refit_mask


def _scene(deformable):
    scene = ol.Scene()
    v, i, n = scenes.uv_sphere(8, 5)
    res = scene.create_mesh(v, i, ol.Material(), normals=n, deformable=deformable)
    inst = scene.add_instances(res, [ol.Transform(np.eye(4, dtype=np.float32))] * 2)
    scene.add_mesh(np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1]], np.float32), np.array([[0, 2, 1]], np.uint32),
                   ol.Material(emission=(4.0, 4.0, 4.0)))
    return scene, res, inst


def test_transform_and_material_edits_keep_every_blas():
    scene, res, inst = _scene(False)
    old = pack_scene(scene)
    m = np.eye(4, dtype=np.float32)
    m[:3, 3] = (1.0, 2.0, 3.0)
    rev = scene.transform_revision
    scene.update_instance_transforms([inst[1]], [ol.Transform(m)])
    assert scene.transform_revision == rev + 1
    scene.update_instance(inst[0], material=ol.Material(base_color=(0.2, 0.3, 0.4)))
    mask = refit_mask(old, pack_scene(scene))
    assert mask is not None and not mask.any()


def test_deformable_mesh_refits_and_rigid_mesh_uploads_again():
    for deformable in (True, False):
        scene, res, inst = _scene(deformable)
        old = pack_scene(scene)
        scene.update_mesh_resource(res, vertices=np.asarray(res.vertices) * 1.1)
        assert inst[0].vertices is res.vertices and inst[0].deformable == deformable
        mask = refit_mask(old, pack_scene(scene))
        if deformable:
            assert mask is not None and mask.tolist() == [1, 0]
        else:
            assert mask is None


def test_topology_or_membership_changes_upload_again():
    scene, res, _inst = _scene(True)
    old = pack_scene(scene)
    idx = np.asarray(res.indices)[:, [0, 2, 1]]
    scene.update_mesh_resource(res, indices=idx)
    assert refit_mask(old, pack_scene(scene)) is None
    scene, res, _inst = _scene(True)
    old = pack_scene(scene)
    scene.add_instance(res)
    assert refit_mask(old, pack_scene(scene)) is None
    scene, res, inst = _scene(True)
    old = pack_scene(scene)
    scene.update_instance(inst[0], visible=False)
    assert refit_mask(old, pack_scene(scene)) is None
