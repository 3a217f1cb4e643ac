"""Generate tests/golden/textures.npz by running the REFERENCE's texture
packing: a scene with three textures (odd sizes, every wrap mode, nearest
and bilinear filters) bound by three materials with KHR texture
transforms, packed by the reference's Scene.texture_data (RGBA8 sRGB and
linear mip pyramids, scene/_core.py:3005-3077), texture_binding_data
(:2983-3003) and the binding indices of triangle_material_data
(:2816-2925).  Imports the reference like make_golden.py does.

Run:  python tests/golden/make_texture_golden.py
"""

from __future__ import annotations

from pathlib import Path
import sys

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import import_reference  # noqa: E402


def build(ol):
    rng = np.random.default_rng(21)
    pixels = [rng.integers(0, 256, (13, 7, 4), dtype=np.uint8), rng.integers(0, 256, (8, 16, 4), dtype=np.uint8),
              rng.integers(0, 256, (5, 9, 4), dtype=np.uint8)]
    textures = [ol.Texture(pixels[0], wrap_s="repeat", wrap_t="mirror", linear_filter=True),
                ol.Texture(pixels[1], wrap_s="clamp", wrap_t="repeat", linear_filter=True),
                ol.Texture(pixels[2], wrap_s="mirror", wrap_t="clamp", linear_filter=False)]
    tf_a = ol.TextureTransform(offset=(0.25, -0.5), scale=(2.0, 0.75), rotation=0.3, texcoord_set=0)
    tf_b = ol.TextureTransform(offset=(0.0, 0.1), scale=(1.5, 1.5), rotation=-1.1, texcoord_set=1)
    materials = [
        ol.Material(base_color=(0.9, 0.8, 0.7), base_color_texture=textures[0], base_color_transform=tf_a,
                    normal_texture=textures[1], normal_scale=0.7),
        ol.Material(metallic_roughness_texture=textures[1], metallic_roughness_transform=tf_b,
                    emissive_texture=textures[2], emission=(1.0, 2.0, 3.0), occlusion_texture=textures[0],
                    occlusion_strength=0.6),
        ol.Material(base_color_texture=textures[2], transmission=0.5, transmission_texture=textures[0],
                    transmission_transform=tf_a),
    ]
    scene = ol.Scene()
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    for k, material in enumerate(materials):
        scene.add_mesh(tri + k, np.array([[0, 1, 2]], np.uint32), material)
    return pixels, scene


def main():
    ol = import_reference()
    pixels, scene = build(ol)
    words = scene.texture_data()
    bindings = scene.texture_binding_data().reshape(-1, 8)
    mats = scene.triangle_material_data().reshape(-1, 12, 4)
    # binding indices per material: base colour, metallic-roughness, emissive,
    # normal (texture_indices), occlusion, transmission (texture_parameters),
    # then normal scale and occlusion strength
    per_material = np.stack([mats[:, 4, 0], mats[:, 4, 1], mats[:, 4, 2], mats[:, 4, 3], mats[:, 5, 1],
                             mats[:, 5, 3], mats[:, 5, 0], mats[:, 5, 2]], axis=1).astype(np.float32)
    np.savez_compressed(HERE / "textures.npz", pixel0=pixels[0], pixel1=pixels[1], pixel2=pixels[2], words=words,
                        bindings=bindings, material_bindings=per_material)
    print("words", words.shape, "bindings", bindings.shape)


if __name__ == "__main__":
    main()
