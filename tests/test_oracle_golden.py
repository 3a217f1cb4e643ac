"""The oracle against the reference's own outputs (tests/golden/, written by
the make_*golden.py scripts from the reference checkout).  CPU only."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import lbvh, reference_path_tracer as ref
from ordinarylight_b200 import packing, scenes


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_scene_mirror_packs_the_reference_triangle_soup(golden):
    data = golden("config1_scene.npz")
    scene, _camera = scenes.box_room()
    tris, colors, emissions = scene.triangles()
    assert tris.shape == (36, 3, 3)
    np.testing.assert_array_equal(tris, data["triangles"])
    np.testing.assert_array_equal(colors, data["colors"])
    np.testing.assert_array_equal(emissions, data["emissions"])
    np.testing.assert_array_equal(scene.triangle_instance_ids(), data["instance_ids"])


def test_emitter_records_match_reference_emissive_triangle_data(golden):
    for name, build in (("config1_scene.npz", lambda: scenes.box_room()[0]),
                        ("spheres_small.npz", lambda: scenes.instanced_spheres(
                            seed=5, instances=2, segments=16, bands=9, emitters=4, extent=3.0)[0])):
        data = golden(name)
        records, weight = packing.emitter_records(build())
        expected = data["emitters"].reshape(-1, 20)
        np.testing.assert_allclose(records, expected, rtol=1e-6, atol=1e-7)
        assert weight == pytest.approx(float(data["emissive_weight"]), rel=1e-12)


def test_oracle_camera_rays_equal_reference_rays(golden):
    data = golden("config1_primary.npz")
    _scene, camera = scenes.box_room()
    origins, directions = ref.camera_rays(camera, 256, 256, np.random.default_rng(1))
    assert _sha(np.ascontiguousarray(directions)) == str(data["directions_f64_sha256"])
    assert _sha(origins.astype(np.float32)) == str(data["origins_sha256"])
    assert _sha(directions.astype(np.float32)) == str(data["directions_sha256"])


def test_oracle_intersect_equals_reference_intersect(golden):
    data = golden("config1_primary.npz")
    scene, camera = scenes.box_room()
    origins, directions = ref.camera_rays(camera, 256, 256, np.random.default_rng(1))
    t, tri = ref.intersect(origins.astype(np.float32), directions.astype(np.float32), scene.triangles()[0])
    np.testing.assert_array_equal(tri, data["triangle"].astype(np.int32))
    np.testing.assert_array_equal(t, data["t"])
    small = golden("spheres_small.npz")
    t2, tri2 = ref.intersect(small["origins"], small["directions"], small["triangles"])
    np.testing.assert_array_equal(tri2, small["triangle"])
    np.testing.assert_array_equal(t2, small["t"])


def test_oracle_render_is_bit_identical_to_reference(golden):
    data = golden("config1_render_small.npz")
    scene, camera = scenes.box_room()
    for frame, key in ((0, "frame0"), (3, "frame3")):
        image = ref.render_frame(scene, camera, 24, 16, samples=2, max_bounces=4, seed=1, frame_index=frame)
        np.testing.assert_array_equal(image, data[key])
    assert np.all(data["frame0"][..., 3] == 0.0)


def test_oracle_volume_render_is_bit_identical_to_reference(golden):
    """The reference's CpuReferenceRenderer on a room with two overlapping
    volumes (emission, clip plane, missing data, log mapping, a mirrored
    nearest transfer function, Henyey-Greenstein single scattering of point,
    spot and directional lights with a second order): the oracle's ray
    march (oracle/reference_volume.py) reproduces its image bit for bit."""
    import parity_scenes

    data = golden("volume_small.npz")
    scene, camera = parity_scenes.volume_room()
    image = ref.render_frame(scene, camera, int(data["width"]), int(data["height"]), samples=int(data["samples"]),
                             max_bounces=int(data["max_bounces"]), seed=int(data["seed"]))
    assert image.tobytes() == data["image"].tobytes()


def test_oracle_counts_closest_hit_rays():
    scene, camera = scenes.box_room()
    counter = ref.RayCounter()
    ref.render_hdr(scene, camera, 8, 8, samples=1, max_bounces=2, seed=1, counter=counter)
    assert counter.rays >= 64 and counter.calls >= 1


def test_oracle_rejects_invalid_sizes():
    scene, camera = scenes.box_room()
    with pytest.raises(ValueError):
        ref.render_hdr(scene, camera, 0, 4)
    with pytest.raises(ValueError):
        ref.render_hdr(scene, camera, 4, 4, samples=0)


def test_morton_codes_are_30_bit_and_stable_order_is_a_permutation():
    tris = np.random.default_rng(3).normal(size=(5000, 3, 3)).astype(np.float32)
    codes = lbvh.morton_codes(tris)
    assert codes.dtype == np.uint32 and int(codes.max()) < (1 << 30)
    order = lbvh.stable_order(codes)
    assert np.array_equal(np.sort(order), np.arange(len(codes)))
    assert np.all(np.diff(codes[order].astype(np.int64)) >= 0)
    # equal keys keep input order
    dup = np.repeat(codes[:10], 3)
    o = lbvh.stable_order(dup)
    for k in range(10):
        assert list(o[3 * k:3 * k + 3]) == sorted(o[3 * k:3 * k + 3])


def test_morton_degenerate_extent_gives_zero_axis():
    tris = np.zeros((4, 3, 3), np.float32)
    tris[:, :, 0] = np.arange(4)[:, None]
    codes = lbvh.morton_codes(tris)
    assert len(set(codes.tolist())) == 4


# ---- participating medium oracle -------------------------------------------------

def test_volume_oracle_trilinear_and_analytic_transmittance():
    from oracle import volume as V

    grid = np.arange(8, dtype=np.float32).reshape(2, 2, 2)   # value = 4z + 2y + x
    corners = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1], [0.5, 0.5, 0.5]])
    assert np.allclose(V.sample_trilinear(grid, corners), [0, 1, 2, 4, 7, 3.5])
    assert np.allclose(V.sample_trilinear(grid, [[-3.0, 2.0, 0.25]]), [0 + 2 + 1.0])   # clipped to the box
    # homogeneous slab of thickness 2 under scale(2): T = exp(-sigma * 2)
    w2b = np.hstack([np.eye(3) * 0.5, np.zeros((3, 1))])
    t = V.transmittance(np.ones((4, 4, 4), np.float32), w2b, 0.8, [[1.0, 1.0, -5.0], [0.5, 1.5, 9.0]],
                        [[0, 0, 1.0], [0, 0, -1.0]])
    assert np.allclose(t, np.exp(-1.6))


def test_volume_oracle_monte_carlo_absorber_matches_analytic():
    from oracle import volume as V

    n = 40000
    w2b = np.hstack([np.eye(3) * 0.5, np.zeros((3, 1))])
    o = np.column_stack([np.full(n, 1.0), np.full(n, 1.0), np.full(n, -5.0)])
    d = np.tile([0.0, 0.0, 1.0], (n, 1))
    rad = V.render_medium(np.ones((4, 4, 4), np.float32), w2b, 0.8, 0.0, o, d, env=[1.0, 1.0, 1.0],
                          max_bounces=2, seed=3)
    expected = np.exp(-1.6)
    assert abs(rad[:, 0].mean() - expected) < 4.0 * np.sqrt(expected * (1 - expected) / n)


def _lights_from_table(ol, table):
    """The lights of analytic_lights.npz's table: rows of (kind, position,
    direction, color, intensity, range (0: none), inner, outer angle), kind 0
    point, 1 directional, 2 spot."""
    lights = []
    for row in table:
        kind = int(row[0])
        pos, direction, color = tuple(row[1:4]), tuple(row[4:7]), tuple(row[7:10])
        intensity, rng_range, inner, outer = float(row[10]), float(row[11]), float(row[12]), float(row[13])
        rng_range = rng_range if rng_range > 0.0 else None
        if kind == 0:
            lights.append(ol.PointLight(position=pos, color=color, intensity=intensity, range=rng_range))
        elif kind == 1:
            lights.append(ol.DirectionalLight(direction=direction, color=color, intensity=intensity))
        else:
            lights.append(ol.SpotLight(position=pos, direction=direction, color=color, intensity=intensity,
                                       inner_cone_angle=inner, outer_cone_angle=outer, range=rng_range))
    return lights


def test_analytic_light_records_match_reference_analytic_light_data(golden):
    """Point, directional and spot lights (ranges, unnormalised directions,
    cone angles) pack to the reference's Scene.analytic_light_data records
    (tests/golden/make_light_golden.py ran the reference on the same lights)."""
    import ordinarylight_b200 as ol

    data = golden("analytic_lights.npz")
    scene = ol.Scene()
    for light in _lights_from_table(ol, data["table"]):
        scene.add_light(light)
    records = packing.light_records(scene)
    assert records.shape == (len(data["table"]), 16)
    np.testing.assert_array_equal(records.reshape(-1, 4, 4), data["records"])
