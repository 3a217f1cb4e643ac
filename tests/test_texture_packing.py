"""Texture packing against the reference's own output (CPU only):
tests/golden/textures.npz holds Scene.texture_data, texture_binding_data
and the per-material binding indices the reference computed for a scene of
three textures and three materials (tests/golden/make_texture_golden.py);
the same scene built with this package must pack to identical words and
records.  The texture sampler oracle is checked on hand-computed cases."""

from __future__ import annotations

from pathlib import Path

import numpy as np

import ordinarylight_b200 as ol
from oracle import textures as otex
from ordinarylight_b200.packing import pack_scene

GOLDEN = Path(__file__).resolve().parent / "golden" / "textures.npz"


def golden_scene(g):
    tex = [ol.Texture(g["pixel0"], wrap_s="repeat", wrap_t="mirror", linear_filter=True),
           ol.Texture(g["pixel1"], wrap_s="clamp", wrap_t="repeat", linear_filter=True),
           ol.Texture(g["pixel2"], wrap_s="mirror", wrap_t="clamp", linear_filter=False)]
    tf_a = ol.TextureTransform(offset=(0.25, -0.5), scale=(2.0, 0.75), rotation=0.3, texcoord_set=0)
    tf_b = ol.TextureTransform(offset=(0.0, 0.1), scale=(1.5, 1.5), rotation=-1.1, texcoord_set=1)
    materials = [
        ol.Material(base_color=(0.9, 0.8, 0.7), base_color_texture=tex[0], base_color_transform=tf_a,
                    normal_texture=tex[1], normal_scale=0.7),
        ol.Material(metallic_roughness_texture=tex[1], metallic_roughness_transform=tf_b, emissive_texture=tex[2],
                    emission=(1.0, 2.0, 3.0), occlusion_texture=tex[0], occlusion_strength=0.6),
        ol.Material(base_color_texture=tex[2], transmission=0.5, transmission_texture=tex[0],
                    transmission_transform=tf_a),
    ]
    scene = ol.Scene()
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    for k, material in enumerate(materials):
        scene.add_mesh(tri + k, np.array([[0, 1, 2]], np.uint32), material)
    return scene


def test_texture_words_bindings_and_material_indices_equal_the_reference():
    g = np.load(GOLDEN)
    packed = pack_scene(golden_scene(g))
    np.testing.assert_array_equal(packed.texture_words, g["words"])
    np.testing.assert_array_equal(packed.texture_bindings, g["bindings"])
    np.testing.assert_array_equal(packed.material_textures[:, :8], g["material_bindings"])
    assert packed.material_textures[1, 8] == 1.0 and packed.material_textures[0, 8] == 0.0   # texcoord set 1 in use


def test_sampler_oracle_known_answers():
    lut = otex.srgb_table()
    assert lut[0] == 0.0 and lut[255] == 1.0 and np.isclose(lut[1], 1.0 / 255.0 / 12.92)
    # a 2x1 texture: texel centres at u = 0.25 and 0.75; halfway is the mean
    px = np.array([[[0, 0, 0, 255], [255, 255, 255, 255]]], np.uint8)
    scene = ol.Scene()
    scene.add_mesh(np.eye(3, dtype=np.float32), np.array([[0, 1, 2]], np.uint32),
                   ol.Material(base_color_texture=ol.Texture(px, wrap_s="clamp", wrap_t="clamp")))
    p = pack_scene(scene)
    uv = np.array([[0.25, 0.5], [0.5, 0.5], [0.75, 0.5], [1.7, 0.5]], np.float32)
    out = otex.sample_material_texture(p.texture_words, p.texture_bindings, 0, uv, uv, False, np.zeros(4, np.float32),
                                       np.zeros(4, np.float32))
    np.testing.assert_allclose(out[:, 0], [0.0, 0.5, 1.0, 1.0], atol=1e-6)
    # a large footprint reads the 1x1 level: the mean colour
    far = otex.sample_material_texture(p.texture_words, p.texture_bindings, 0, uv[:1], uv[:1], False,
                                       np.array([10.0], np.float32), np.array([10.0], np.float32))
    np.testing.assert_allclose(far[0, 0], 128.0 / 255.0, atol=1e-6)
