"""Material textures on the device against the restated reference lookups
(oracle/textures.py, oracle/pbr.py): the sampler alone on every binding of
the reference-packed golden scene (wrap modes, filters, KHR transforms,
sRGB decode, ray-cone LOD and trilinear blending), a textured emitter seen
by camera rays, and base-colour, metallic-roughness and normal maps under
a directional light, where every pixel is a deterministic direct term."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import ordinarylight_b200 as ol
from oracle import pbr
from oracle import textures as otex
from oracle.dielectric import _hits
from ordinarylight_b200 import CudaWavefrontRenderer
from ordinarylight_b200.packing import pack_scene

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "textures.npz"


def test_sampler_matches_the_restated_lookup(native_library, cuda_device):
    from test_texture_packing import golden_scene

    scene = golden_scene(np.load(GOLDEN))
    packed = pack_scene(scene)
    rng = np.random.default_rng(5)
    n = 4096
    uv0 = rng.uniform(-3.0, 3.0, (n, 2)).astype(np.float32)
    uv1 = rng.uniform(-3.0, 3.0, (n, 2)).astype(np.float32)
    fp = np.where(rng.random(n) < 0.25, 0.0, np.exp(rng.uniform(np.log(1e-3), np.log(3.0), n))).astype(np.float32)
    fp1 = fp[::-1].copy()
    with CudaWavefrontRenderer() as r:
        for binding in range(len(packed.texture_bindings)):
            for srgb in (False, True):
                got = r.sample_texture(scene, binding, uv0, uv1, fp, fp1, srgb=srgb)
                want = otex.sample_material_texture(packed.texture_words, packed.texture_bindings, binding, uv0, uv1,
                                                    srgb, fp, fp1)
                # float32 blends: the device may fuse multiply-adds, numpy does not
                np.testing.assert_allclose(got, want, atol=1e-5, rtol=0)


def _textured_floor(material_args, uv_scale=0.1):
    scene = ol.Scene()
    v = np.array([[-30, 0, -30], [-30, 0, 30], [30, 0, 30], [30, 0, -30]], np.float32)
    res = scene.create_mesh(v, np.array([[0, 1, 2], [0, 2, 3]], np.uint32), ol.Material(**material_args),
                            normals=np.tile([0.0, 1.0, 0.0], (4, 1)).astype(np.float32),
                            texcoords=v[:, [0, 2]] * uv_scale)
    scene.add_instance(res)
    scene.set_environment(ol.EnvironmentLight(color=(0.0, 0.0, 0.0), intensity=0.0))
    camera = ol.PerspectiveCamera(position=(0.3, 4.0, -7.0), target=(0.0, 0.0, 1.0), vertical_fov_degrees=45.0)
    return scene, camera


def _hit_uv(r, scene, camera, w, h):
    """The oracle's hits of the device's camera rays: points, view vectors,
    interpolated texcoords and which pixels are away from triangle edges."""
    o, d = r.camera_rays(camera, w, h, sample=0, frame_index=0)
    o, d = np.asarray(o, np.float64), np.asarray(d, np.float64)
    tris = np.array([m.world_vertices[m.indices] for m in scene.visible_meshes]).reshape(-1, 3, 3)
    uvs = np.array([m.texcoords[m.indices] for m in scene.visible_meshes]).reshape(-1, 3, 2)
    t, k, bu, bv = _hits(o, d, tris)
    hit = k >= 0
    kk = np.maximum(k, 0)
    w0 = 1.0 - bu - bv
    uv = uvs[kk, 0] * w0[:, None] + uvs[kk, 1] * bu[:, None] + uvs[kk, 2] * bv[:, None]
    edge = np.minimum(np.minimum(bu, bv), w0) < 1e-4
    return o + d * t[:, None], -d, uv.astype(np.float32), hit & ~edge


def _texture(rng, h, w):
    px = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    px[..., 3] = 255
    return px


def test_textured_emission_seen_by_camera_rays(native_library, cuda_device):
    rng = np.random.default_rng(8)
    tex = ol.Texture(_texture(rng, 12, 10), wrap_s="mirror", wrap_t="repeat")
    tf = ol.TextureTransform(offset=(0.3, 0.1), scale=(1.3, 0.8), rotation=0.4)
    scene, camera = _textured_floor(dict(base_color=(0.0, 0.0, 0.0), emission=(2.0, 1.5, 1.0), emissive_texture=tex,
                                         emissive_transform=tf, emission_two_sided=True))
    w, h = 64, 48
    with CudaWavefrontRenderer(max_bounces=1, samples_per_pixel=1) as r:
        img = r.render_frame(scene, camera, w, h, frame_index=0)
        _p, _view, uv, ok = _hit_uv(r, scene, camera, w, h)
    packed = pack_scene(scene)
    zero = np.zeros(len(uv), np.float32)
    texel = otex.sample_material_texture(packed.texture_words, packed.texture_bindings, 0, uv, uv, True, zero, zero)
    expected = texel[:, :3] * np.array([2.0, 1.5, 1.0], np.float32)
    assert ok.mean() > 0.5
    np.testing.assert_allclose(img[..., :3].reshape(-1, 3)[ok], expected[ok], rtol=2e-4, atol=2e-5)


def test_base_metallic_roughness_and_normal_maps_under_a_directional_light(native_library, cuda_device):
    rng = np.random.default_rng(9)
    base_px = _texture(rng, 16, 16)
    mr_px = _texture(rng, 8, 8)
    n = rng.normal(size=(16, 16, 3)) * np.array([0.35, 0.35, 0.0]) + np.array([0.0, 0.0, 1.0])
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    normal_px = np.concatenate([np.round((n * 0.5 + 0.5) * 255.0), np.full((16, 16, 1), 255.0)], -1).astype(np.uint8)
    normal_tf = ol.TextureTransform(scale=(1.5, 1.2), rotation=0.6)
    material = dict(base_color=(0.9, 0.8, 0.7), roughness=0.8, metallic=0.6,
                    base_color_texture=ol.Texture(base_px), metallic_roughness_texture=ol.Texture(mr_px),
                    normal_texture=ol.Texture(normal_px), normal_scale=0.8, normal_transform=normal_tf)
    scene, camera = _textured_floor(material)
    light = ol.DirectionalLight(direction=(-0.3, -1.0, 0.4), color=(1.0, 0.9, 0.8), intensity=3.0)
    scene.add_light(light)
    w, h = 64, 48
    with CudaWavefrontRenderer(max_bounces=2, samples_per_pixel=1) as r:
        img = r.render_frame(scene, camera, w, h, frame_index=0)
        _p, view, uv, ok = _hit_uv(r, scene, camera, w, h)
    packed = pack_scene(scene)
    words, bindings, mats = packed.texture_words, packed.texture_bindings, packed.material_textures[0]
    zero = np.zeros(len(uv), np.float32)
    base = otex.sample_material_texture(words, bindings, int(mats[0]), uv, uv, True, zero, zero)[:, :3] * \
        np.array([0.9, 0.8, 0.7], np.float32)
    mr = otex.sample_material_texture(words, bindings, int(mats[1]), uv, uv, False, zero, zero)
    roughness, metallic = 0.8 * mr[:, 1], 0.6 * mr[:, 2]
    sampled = otex.sample_material_texture(words, bindings, int(mats[3]), uv, uv, False, zero, zero)
    rec = bindings[int(mats[3])]
    ns = np.tile([0.0, 1.0, 0.0], (len(uv), 1))
    tangent = np.tile(packed.tangents[0], (len(uv), 1)).astype(np.float64)
    nm = otex.apply_normal(sampled.astype(np.float64), 0.8, ns, tangent, rec[1], rec[2], rec[6], rec[7])
    nm = np.where((np.sum(nm * ns, axis=1) < 0.0)[:, None], -nm, nm)
    expected = pbr.directional_radiance(base, roughness, metallic, nm, view, light.direction, light.color,
                                        light.intensity)
    assert ok.mean() > 0.5
    np.testing.assert_allclose(img[..., :3].reshape(-1, 3)[ok], expected[ok], rtol=3e-3, atol=2e-5)


def test_textured_and_untextured_scenes_mix_in_one_batch(native_library, cuda_device):
    """A run with a textured scene uses the textured kernel variants for all
    of its jobs; an untextured job's image must still equal its plain frame
    (rendered with the untextured variants) bit for bit."""
    from ordinarylight_b200 import scenes
    from ordinarylight_b200.renderers.cuda import RenderRequest

    rng = np.random.default_rng(3)
    tex = ol.Texture(_texture(rng, 16, 16))
    textured, tcam = _textured_floor(dict(base_color=(0.9, 0.9, 0.9), roughness=0.6, base_color_texture=tex))
    textured.set_environment(ol.EnvironmentLight(color=(0.6, 0.7, 0.9), intensity=1.0))
    plain_scene, pcam = scenes.instanced_spheres(seed=7, instances=6, segments=24, bands=13, emitters=32,
                                                 extent=5.0)
    reqs = [RenderRequest(textured, tcam, 48, 40, samples=2, frame_index=1, max_bounces=4),
            RenderRequest(plain_scene, pcam, 64, 48, samples=2, frame_index=2, max_bounces=4)]
    for restir in (False, True):
        with CudaWavefrontRenderer(max_bounces=4, restir=restir) as r:
            batch = r.render_batch(reqs)
        for req, img in zip(reqs, batch):
            with CudaWavefrontRenderer(max_bounces=4, restir=restir) as p:
                ref = p.render_frame(req.scene, req.camera, req.width, req.height, samples=req.samples,
                                     frame_index=req.frame_index)
            assert img.tobytes() == ref.tobytes()
