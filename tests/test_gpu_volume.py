"""Participating medium: CUDA delta tracking against the oracle.

* a homogeneous pure absorber seen through a slab of constant thickness
  transmits exp(-sigma_t d) of the environment, the analytic answer;
* a heterogeneous (fBm) absorber transmits exp(-optical depth) per pixel,
  integrated by the oracle's fine midpoint rule over the same grid with the
  reference's trilinear lookup;
* a scattering medium (albedo 0.9, isotropic) under a constant environment
  and a directional light agrees with the oracle's independent Monte Carlo
  estimator in image mean and per pixel;
* a medium over a surface renders the same bits in plain and batched form.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import volume as V
from ordinarylight_b200 import CudaWavefrontRenderer, scene as m, scenes
from ordinarylight_b200.renderers.cuda import RenderRequest

pytestmark = pytest.mark.gpu

BOX = m.Transform.scale((2.0, 2.0, 2.0))          # the unit box scaled to [0, 2]^3
W2B = np.linalg.inv(BOX.matrix.astype(np.float64))[:3, :4]


def medium_scene(grid, sigma, albedo, *, env=1.0, sun=None):
    s = m.Scene()
    s.add_volume(grid, m.VolumeMaterial(sigma_t_scale=sigma, albedo=albedo), transform=BOX)
    s.set_environment(m.EnvironmentLight(color=(1.0, 1.0, 1.0), intensity=env))
    if sun is not None:
        s.add_light(m.DirectionalLight(direction=sun, color=(1.0, 1.0, 1.0), intensity=3.0))
    return s


# orthographic camera looking down +z through the box, framing x, y in [0.5, 1.5]
ORTHO = m.OrthographicCamera(position=(1.0, 1.0, -4.0), target=(1.0, 1.0, 0.0), vertical_size=1.0)


def ortho_rays(width, height, sub):
    """Sub-pixel grid of the orthographic camera's rays (x right, y up)."""
    js = (np.arange(sub) + 0.5) / sub
    xs = ((np.arange(width)[:, None] + js[None, :]) / width).reshape(-1)
    ys = ((np.arange(height)[:, None] + js[None, :]) / height).reshape(-1)
    # ndc: x in [-1, 1] left to right, y flipped; half extents 0.5 (square image)
    px = 1.0 - (xs * 2.0 - 1.0) * 0.5   # the camera's right vector is -x when looking down +z
    py = 1.0 + (1.0 - ys * 2.0) * 0.5
    gx, gy = np.meshgrid(px, py)
    o = np.column_stack([gx.ravel(), gy.ravel(), np.full(gx.size, -4.0)])
    d = np.tile([0.0, 0.0, 1.0], (gx.size, 1))
    return o, d


def test_homogeneous_absorber_is_analytic(native_library, cuda_device):
    scene = medium_scene(np.ones((4, 4, 4), np.float32), 0.8, 0.0)
    with CudaWavefrontRenderer(max_bounces=1, seed=1) as r:
        img = r.render_frame(scene, ORTHO, 64, 64, samples=16)
        assert r.last_timings["traversal_errors"] == 0
    expected = float(np.exp(-0.8 * 2.0))
    n = 64 * 64 * 16
    assert np.allclose(img[..., 0], img[..., 1]) and np.allclose(img[..., 0], img[..., 2])
    assert abs(float(img[..., 0].mean()) - expected) < 4.0 * np.sqrt(expected * (1 - expected) / n)


def test_heterogeneous_absorber_matches_ray_march(native_library, cuda_device):
    grid = scenes.fbm_volume(24, seed=11)
    sigma, w, spp, sub = 2.0, 24, 256, 4
    scene = medium_scene(grid, sigma, 0.0)
    with CudaWavefrontRenderer(max_bounces=1, seed=2) as r:
        img = r.render_frame(scene, ORTHO, w, w, samples=spp)[..., 0].astype(np.float64)
    o, d = ortho_rays(w, w, sub)
    t = V.transmittance(grid, W2B, sigma, o, d, steps=512).reshape(w, sub, w, sub)
    expected = t.mean(axis=(1, 3))
    assert 0.05 < expected.mean() < 0.95 and expected.std() > 0.02    # a genuinely varying medium
    se = np.sqrt(np.maximum(expected * (1 - expected), 1e-4) / spp)
    z = (img - expected) / se
    assert abs(img.mean() - expected.mean()) < 4.0 * np.sqrt(np.mean(se * se) / img.size)
    assert np.mean(z * z) < 1.5


def test_scattering_medium_matches_monte_carlo_oracle(native_library, cuda_device):
    grid = scenes.fbm_volume(16, seed=13)
    sigma, albedo, w, bounces = 2.5, 0.9, 16, 4
    sun = (0.3, -1.0, 0.4)
    scene = medium_scene(grid, sigma, albedo, env=0.5, sun=sun)
    spp_gpu, spp_cpu = 2048, 256
    with CudaWavefrontRenderer(max_bounces=bounces, seed=3, russian_roulette_start=0) as r:
        gpu = r.render_frame(scene, ORTHO, w, w, samples=spp_gpu)[..., 0].astype(np.float64)
        assert r.last_timings["shadow_rays"] > 0
    o, d = ortho_rays(w, w, 16)                                        # 256 jittered-free sub-rays per pixel
    rad = V.render_medium(grid, W2B, sigma, albedo, o, d, env=[0.5] * 3, light_dir=sun, light_rgb=[3.0] * 3,
                          max_bounces=bounces, seed=5)[:, 0].reshape(w, 16, w, 16)
    cpu = rad.mean(axis=(1, 3))
    cpu_se = rad.std(axis=(1, 3)) / np.sqrt(spp_cpu)
    # GPU per-pixel SE estimated from the CPU sample spread at the GPU's spp
    gpu_se = rad.std(axis=(1, 3)) / np.sqrt(spp_gpu)
    se = np.sqrt(cpu_se ** 2 + gpu_se ** 2) + 1e-6
    assert abs(gpu.mean() - cpu.mean()) < 4.0 * np.sqrt(np.mean(se ** 2) / gpu.size) + 2e-3 * cpu.mean()
    z = (gpu - cpu) / se
    assert np.mean(z * z) < 2.0


def test_medium_over_terrain_plain_equals_batch(native_library, cuda_device):
    scene, camera = scenes.terrain(size=64, volume_size=16)
    req = RenderRequest(scene, camera, 48, 32, samples=2, frame_index=4, max_bounces=5)
    with CudaWavefrontRenderer(max_bounces=5, seed=1) as r:
        plain = r.render_frame(scene, camera, 48, 32, samples=2, frame_index=4)
        again = r.render_frame(scene, camera, 48, 32, samples=2, frame_index=4)
        batch = r.render_batch([req])[0]
        assert r.last_timings["traversal_errors"] == 0
    assert np.all(np.isfinite(plain)) and float(plain[..., :3].mean()) > 0.0
    assert plain.tobytes() == again.tobytes() == batch.tobytes()
