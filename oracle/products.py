"""ORACLE — test infrastructure only, never part of the product path.

numpy restatement of the reference's host-side product arithmetic of
render_wavefront_outputs (ordinarylight/targets/vulkan/api.py):

* ``sample_variance``  the ``variance`` product (:1404-1431): per-sample
  luminance r*0.2126 + g*0.7152 + b*0.0722 in float32, sums of l and l^2 in
  float64 in sample order, (sum l^2 - (sum l)^2 / n) / (n - 1) clamped at 0,
  zeros for one sample.
* ``project_positions``  _project_positions (:1118-1136).
* ``motion_product``  _motion_product (:1151-1200): for hits on meshes whose
  topology and vertex count are unchanged since the captured frame (matched
  by Mesh.id), the old world point is the old triangle's vertices weighted
  by the barycentrics (1 - u - v, u, v) under the old transform, and the
  motion is its projection now minus its projection under the old camera.
"""

from __future__ import annotations

import numpy as np


def sample_variance(per_sample):
    lum_sum = lum_sq = None
    for radiance in per_sample:
        lum = (radiance[..., 0] * 0.2126 + radiance[..., 1] * 0.7152 + radiance[..., 2] * 0.0722).astype(np.float64)
        if lum_sum is None:
            lum_sum, lum_sq = lum, lum * lum
        else:
            lum_sum = lum_sum + lum
            lum_sq = lum_sq + lum * lum
    n = len(per_sample)
    if n == 1:
        return np.zeros(per_sample[0].shape[:2], np.float32)
    return np.maximum((lum_sq - lum_sum * lum_sum / n) / (n - 1), 0.0).astype(np.float32)


def project_positions(positions, camera, width, height):
    origin = np.asarray(camera.position, np.float64)
    forward = np.asarray(camera.target, np.float64) - origin
    forward /= np.linalg.norm(forward)
    right = np.cross(forward, np.asarray(camera.up, np.float64))
    right /= np.linalg.norm(right)
    up = np.cross(right, forward)
    relative = np.asarray(positions, np.float64) - origin
    distance = relative @ forward
    scale = np.tan(np.radians(camera.vertical_fov_degrees) * 0.5)
    safe = np.maximum(distance, 1e-12)
    ndc_x = (relative @ right) / (safe * scale * (width / height))
    ndc_y = -(relative @ up) / (safe * scale)
    return np.column_stack(((ndc_x + 1.0) * 0.5 * width, (ndc_y + 1.0) * 0.5 * height)), distance > 1e-8


def capture_state(scene, camera, size):
    """The captured frame: camera, size and each visible mesh's arrays."""
    return {"scene": scene, "camera": camera, "size": size,
            "meshes": {m.id: (np.array(m.vertices), np.array(m.indices), np.array(m.transform.matrix))
                       for m in scene.visible_meshes}}


def motion_product(previous, scene, camera, width, height, primitive, position, barycentric):
    motion = np.zeros((height, width, 2), np.float32)
    if previous is None or previous["scene"] is not scene or previous["size"] != (width, height):
        return motion
    flat_prim = primitive.reshape(-1)
    flat_pos = position.reshape((-1, 3))
    flat_bary = barycentric.reshape((-1, 2))
    flat_motion = motion.reshape((-1, 2))
    offset = 0
    for mesh in scene.visible_meshes:
        count = len(mesh.indices)
        selected = np.flatnonzero((flat_prim >= offset) & (flat_prim < offset + count))
        old = previous["meshes"].get(mesh.id)
        if selected.size and old is not None:
            old_vertices, old_indices, old_transform = old
            if (old_indices.shape == mesh.indices.shape and np.array_equal(old_indices, mesh.indices)
                    and old_vertices.shape == mesh.vertices.shape):
                local = flat_prim[selected].astype(np.int64) - offset
                tris = old_vertices[old_indices[local]]
                uv = flat_bary[selected]
                w = np.column_stack((1.0 - uv[:, 0] - uv[:, 1], uv[:, 0], uv[:, 1]))
                old_object = np.sum(tris * w[..., None], axis=1)
                old_world = old_object @ old_transform[:3, :3].T + old_transform[:3, 3]
                cur, cur_ok = project_positions(flat_pos[selected], camera, width, height)
                was, was_ok = project_positions(old_world, previous["camera"], width, height)
                ok = cur_ok & was_ok
                flat_motion[selected[ok]] = (cur[ok] - was[ok]).astype(np.float32)
        offset += count
    return motion
