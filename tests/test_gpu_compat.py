"""Reference-compatible mode beyond the closed-box room, against images the
reference itself rendered (tests/golden/make_volume_golden.py runs the
reference's CpuReferenceRenderer / ReferencePathTracer):

* the reference's volume model (ordinarylight/volume/_core.py:252-504, the
  ray march every segment of ReferencePathTracer.render_hdr crosses,
  renderers/reference/path_tracer.py:55-65): ray by ray against the oracle's
  restatement on the renderer's own camera rays, then converged images of
  the volume room (two overlapping media, clip plane, missing data,
  Henyey-Greenstein phase, two scattering orders, point, spot and
  directional lights);
* configs 2 and 3 scaled for the reference's brute-force intersector
  (4 instances of a 1,280-triangle sphere with 16 emitters; a 32 x 32 fBm
  terrain with a sun-lit 24^3 medium): converged images;
* a scene packed from the reference's own objects renders exactly like the
  same scene built with this package's scene model.

Tolerance (north star): per-channel image means within 3 standard errors and
relative RMSE below 1 % once both sides' Monte Carlo noise is removed.
"""

from __future__ import annotations

import numpy as np
import pytest

from image_parity import batch_estimate, compare
import parity_scenes
from oracle import reference_path_tracer as ref
from oracle import reference_volume
from ordinarylight_b200 import CudaWavefrontRenderer
from ordinarylight_b200.packing import PackedScene

pytestmark = pytest.mark.gpu


def test_volume_march_matches_the_oracle_ray_by_ray(native_library, cuda_device):
    """One segment per pixel (max_bounces 1) on the renderer's own camera
    rays: radiance = volume radiance + transmittance x (emission or sky),
    the march in float32 against the oracle's float64 sums."""
    scene, camera = parity_scenes.volume_room()
    w, h = 24, 16
    with CudaWavefrontRenderer(mode="reference_compatible", max_bounces=1) as r:
        img = r.render_frame(scene, camera, w, h, samples=1)
        o, d = r.camera_rays(camera, w, h, sample=0, frame_index=0)
    tris, _colors, emissions = scene.triangles()
    t, tri = ref.intersect(o.astype(np.float32), d.astype(np.float32), tris)
    vols = scene.visible_volumes
    entries, exits = reference_volume.intersect_unit_boxes(o, d, vols)
    vol_rad, vol_t = reference_volume.integrate_volumes(vols, o, d, entries, exits, max_distance=t,
                                                        lights=scene.lights)
    surface = np.where((tri >= 0)[:, None], emissions[np.maximum(tri, 0)], ref.sky(d, scene.environment))
    expected = vol_rad + vol_t[:, None] * surface
    assert np.count_nonzero(vol_t < 0.999) >= 32                # the media are in view
    np.testing.assert_allclose(img[..., :3].reshape(-1, 3), expected, rtol=2e-3, atol=2e-5)


CONVERGED = {"volume_room": (parity_scenes.volume_room, 3), "scaled_instanced": (parity_scenes.scaled_instanced, 4),
             "scaled_terrain": (parity_scenes.scaled_terrain, 4)}


@pytest.mark.parametrize("name", list(CONVERGED))
def test_reference_compatible_mode_converges_to_the_reference(native_library, cuda_device, golden, name):
    data = golden(f"compat_{name}.npz")
    builder, bounces = CONVERGED[name]
    scene, camera = builder()
    w, h = int(data["width"]), int(data["height"])
    assert bounces == int(data["max_bounces"])
    with CudaWavefrontRenderer(mode="reference_compatible", max_bounces=bounces) as r:
        gpu = batch_estimate(np.stack([r.render_frame(scene, camera, w, h, samples=2048, frame_index=10 + k)[..., :3]
                                       for k in range(16)]))
    batches = data["batch_means"]
    ref_image_se = batches.std(axis=0, ddof=1) / np.sqrt(len(batches))
    compare(data["mean"], data["sem"], ref_image_se, *gpu, tolerance=0.01, label=name)


@pytest.mark.parametrize("mode", ["reference_compatible", "production"])
def test_a_scene_packed_from_reference_objects_renders_like_the_mirror_scene(native_library, cuda_device, golden,
                                                                             mode):
    """tests/golden/refpacked_scaled_terrain.npz was packed from the scaled
    config-3 scene built with the reference's own Scene API."""
    from conftest import GOLDEN

    packed = PackedScene.load(GOLDEN / "refpacked_scaled_terrain.npz")
    scene, camera = parity_scenes.scaled_terrain()
    with CudaWavefrontRenderer(mode=mode, max_bounces=3) as r:
        a = r.render_frame(packed, camera, 24, 16, samples=4, frame_index=3)
    with CudaWavefrontRenderer(mode=mode, max_bounces=3) as r:
        b = r.render_frame(scene, camera, 24, 16, samples=4, frame_index=3)
    assert a.tobytes() == b.tobytes()
