"""Production estimator against the production-transport oracle.

The CUDA renderer's production mode (GGX + Lambert BSDF, one-sample
next-event estimation with power-heuristic MIS, Russian roulette, ReSTIR DI)
must converge to the image of oracle/transport.c, a CPU restatement of the
reference GPU wavefront's transport (shaders/transport_v1/lighting.glsl:
137-404, 618-678; shaders/ordinaryshade_primary.glsl:506-609, 668-734;
shaders/wavefront_shade.comp:331-348, 412-440, 569-580) with its own
hierarchy, random numbers and estimator structure (all analytic lights per
vertex, a CDF-selected area sample and environment next-event estimation).
The oracle's images are fixtures (tests/golden/production_*.npz, made by
tests/golden/make_production_golden.py at 8,192 or 32,768 samples per pixel).

Tolerance (north star): per-channel image means within 3 standard errors and
noise-corrected relative RMSE below 1 %.
"""

from __future__ import annotations

import numpy as np
import pytest

from image_parity import batch_estimate, compare, oracle_image_se
import parity_scenes
from ordinarylight_b200 import CudaWavefrontRenderer

pytestmark = pytest.mark.gpu

BATCHES = 16


def _oracle(golden, name):
    data = golden(f"production_{name}.npz")
    sem = data["sem"].astype(np.float64)
    return data["mean"].astype(np.float64), sem, oracle_image_se(sem)


def _render_batches(name, spp, **config):
    case = parity_scenes.CASES[name]
    scene, camera = parity_scenes.build(name)
    w, h = case["size"]
    settings = dict(max_bounces=case["max_bounces"], russian_roulette_start=case["rr_start"],
                    russian_roulette_min_survival=case["rr_min"])
    settings.update(config)
    with CudaWavefrontRenderer(**settings) as r:
        return np.stack([r.render_frame(scene, camera, w, h, samples=spp, frame_index=100 + k)[..., :3]
                         for k in range(BATCHES)])


PLAIN = [n for n in parity_scenes.CASES if n != "restir_spheres"]


@pytest.mark.parametrize("name", PLAIN)
def test_production_estimator_matches_the_oracle(native_library, cuda_device, golden, name):
    """Box room and the roughness {0.05, 0.5, 1} x metallic {0, 1} sweep of
    two GGX spheres (area emitters, a point light, the analytic sky)."""
    gpu = batch_estimate(_render_batches(name, 1024))
    compare(*_oracle(golden, name), *gpu, tolerance=0.01, label=name)


@pytest.mark.parametrize("name", ["ggx_r0.5_m0", "ggx_r1_m1"])
def test_pure_bsdf_sampling_matches_the_oracle(native_library, cuda_device, golden, name):
    """Without next-event estimation the same image comes from BSDF sampling
    alone (emitters and sky reached by the sampled directions; the point
    light, a delta light, then contributes nothing, so the scene is rendered
    without it).  Near-mirror surfaces are left out here: BSDF sampling of
    their small emitter reflections is too heavy-tailed for a per-pixel
    error bound at test sample counts (their production estimator, with
    next-event estimation, is compared above)."""
    case = parity_scenes.CASES[name]
    scene, camera = parity_scenes.build(name)
    for light in list(scene.lights):
        scene.lights.remove(light)
    w, h = case["size"]
    with CudaWavefrontRenderer(max_bounces=case["max_bounces"], russian_roulette_start=case["rr_start"],
                               nee=False) as r:
        gpu = batch_estimate(np.stack([r.render_frame(scene, camera, w, h, samples=2048, frame_index=k)[..., :3]
                                       for k in range(BATCHES)]))
    from oracle import production

    mean, sem = production.render(scene, camera, w, h, samples=4096, max_bounces=case["max_bounces"],
                                  rr_start=case["rr_start"], seed=5)
    compare(mean, sem, oracle_image_se(sem), *gpu, tolerance=0.01, label=name + " without NEE")


def _restir_sequences(name, sequences, frames, spp, temporal):
    """Mean image of `sequences` independent ReSTIR frame sequences (one
    renderer, hence one history, per sequence; seeds differ), each of
    `frames` consecutive frames, as K = `sequences` independent batches."""
    case = parity_scenes.CASES[name]
    scene, camera = parity_scenes.build(name)
    w, h = case["size"]
    out = []
    for k in range(sequences):
        with CudaWavefrontRenderer(max_bounces=case["max_bounces"], russian_roulette_start=case["rr_start"],
                                   russian_roulette_min_survival=case["rr_min"], restir=True,
                                   restir_temporal=temporal, seed=1 + 7919 * k) as r:
            out.append(np.mean([r.render_frame(scene, camera, w, h, samples=spp, frame_index=f)[..., :3]
                                for f in range(frames)], axis=0))
    return np.stack(out)


@pytest.mark.parametrize("temporal", [True, False])
def test_restir_converges_to_the_oracle(native_library, cuda_device, golden, temporal):
    """ReSTIR DI (32 candidates, temporal history when on, one spatial pass
    of 5 neighbours in 30 px) on the 64-emitter instanced scene: the average
    of 16 independent 16-frame sequences against the oracle's 32,768-spp
    image, at the north star's 1 %."""
    gpu = batch_estimate(_restir_sequences("restir_spheres", 16, 16, 32, temporal))
    compare(*_oracle(golden, "restir_spheres"), *gpu, tolerance=0.01,
            label=f"ReSTIR temporal={temporal}")


def test_restir_with_analytic_lights_matches_the_oracle(native_library, cuda_device, golden):
    """A ReSTIR frame whose scene also has an analytic light: the primary
    vertex chooses between the reservoir's emitter sample and an analytic
    light, so neither kind of light is lost."""
    gpu = batch_estimate(_restir_sequences("ggx_r0.5_m0", 16, 8, 128, True))
    compare(*_oracle(golden, "ggx_r0.5_m0"), *gpu, tolerance=0.01, label="ReSTIR with a point light")
