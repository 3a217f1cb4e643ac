"""The drop-in boundary with the reference's own objects, on CPU.

Where a reference checkout is present (a ``reference`` directory beside this
repository, or OL_REFERENCE_ROOT), the reference package is imported with
stubs for its three un-vendored dependencies (tests/golden/make_golden.py)
and:

* its ``ordinarylight.Scene`` objects flatten to exactly the arrays the same
  scenes built with this package's mirror of the scene model give: the box
  room, instanced spheres, lights of every kind, a textured mesh and volumes
  in the reference's volume model;
* ``CudaWavefrontRenderer`` satisfies the reference's runtime-checkable
  ``RendererProtocol`` and its product and resident-scene extensions
  (ordinarylight/renderers/base.py:42-112);
* the reference's own facade ``ordinarylight.Renderer(implementation=...)``
  (ordinarylight/renderer/_core.py:221-251) drives it: frame indices,
  ``reset_sequence`` and the HDR contract hold, and the scene description
  that reaches the C ABI is the one packed from the reference scene.

The renderer runs here against a stand-in for the C library (no GPU): only
the Python side of the boundary is under test; tests/test_gpu_*.py render.
"""

from __future__ import annotations

import ctypes
from dataclasses import fields
from pathlib import Path
import sys

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.skipif(not make_golden.reference_available(),
                                reason="no OrdinaryLight checkout beside this repository (OL_REFERENCE_ROOT)")


@pytest.fixture(scope="module")
def ref_ol():
    return make_golden.import_reference()


def _textured(m):
    scene = m.Scene()
    rng = np.random.default_rng(4)
    tex = m.Texture(rng.integers(0, 256, (8, 8, 4), dtype=np.uint8), wrap_s="repeat", wrap_t="mirror")
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    uv = np.array([[0, 0], [2, 0], [2, 2], [0, 2]], np.float32)
    scene.add_mesh(v, np.array([[0, 1, 2], [0, 2, 3]], np.uint32),
                   m.Material(base_color_texture=tex, roughness=0.3), texcoords=uv)
    return scene


def _lights(m):
    import parity_scenes

    scene, _ = parity_scenes.ggx_pair(0.5, 1.0, m)
    scene.add_light(m.SpotLight(position=(0, 3, 0), direction=(0, -1, 0.2), intensity=5.0, inner_cone_angle=0.2,
                                outer_cone_angle=0.6, range=9.0))
    scene.add_light(m.DirectionalLight(direction=(0.2, -1.0, 0.1), color=(1.0, 0.8, 0.6), intensity=2.0))
    scene.set_environment(m.EnvironmentLight(color=(0.3, 0.4, 0.5), intensity=1.5))
    return scene


def _builders():
    import parity_scenes
    from ordinarylight_b200 import scenes

    return {
        "box_room": lambda m: scenes.box_room(m)[0],
        "instanced": lambda m: parity_scenes.scaled_instanced(m)[0],
        "lights": _lights,
        "textured": _textured,
        "volume_room": lambda m: parity_scenes.volume_room(m)[0],
        "scaled_terrain": lambda m: parity_scenes.scaled_terrain(m)[0],
    }


def _same(a, b):
    if isinstance(a, dict) or isinstance(b, dict):
        return a is not None and b is not None and a.keys() == b.keys() and all(_same(a[k], b[k]) for k in a)
    if isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
        a, b = np.asarray(a), np.asarray(b)
        return a.dtype == b.dtype and a.shape == b.shape and a.tobytes() == b.tobytes()
    return a == b


@pytest.mark.parametrize("name", list(_builders()))
def test_reference_scenes_pack_like_the_mirror(ref_ol, name):
    import ordinarylight_b200 as mirror
    from ordinarylight_b200.packing import PackedScene, pack_scene

    build = _builders()[name]
    ref_packed = pack_scene(build(ref_ol))
    mine = pack_scene(build(mirror))
    for f in fields(PackedScene):
        if f.name == "mesh_sources":
            continue
        assert _same(getattr(ref_packed, f.name), getattr(mine, f.name)), f"{name}: field {f.name} differs"


class _StandInLibrary:
    """The C entry points the renderer's render path calls, in Python: keeps
    the uploaded scene description and fills the output with the frame
    index."""

    def __init__(self):
        self.uploads = []
        self.renders = []

    def olc_create(self, config, handle):
        handle._obj.value = 1
        return 0

    def olc_destroy(self, ctx):
        return 0

    def olc_last_error(self, ctx):
        return b""

    def olc_upload_scene(self, ctx, desc):
        d = desc._obj
        self.uploads.append(dict(meshes=d.num_meshes, instances=d.num_instances, materials=d.num_materials,
                                 emitters=d.num_emitters, lights=d.num_lights, ref_volumes=d.num_ref_volumes))
        return 0

    def olc_reset_history(self, ctx):
        self.resets = getattr(self, "resets", 0) + 1
        return 0

    def olc_render(self, ctx, camera, width, height, spp, frame_index, out, on_device, stats):
        values = np.full(width * height * 4, float(frame_index), np.float32)
        ctypes.memmove(out, values.ctypes.data, values.nbytes)
        s = stats._obj
        s.camera_rays = width * height * spp
        s.gpu_ms = 1.0
        self.renders.append((width, height, spp, frame_index))
        return 0


@pytest.fixture
def stand_in(monkeypatch):
    from ordinarylight_b200 import _native

    from ordinarylight_b200.renderers import cuda

    lib = _StandInLibrary()
    monkeypatch.setattr(_native, "load", lambda: lib)
    # page-locked host frames need a driver; plain arrays stand in
    monkeypatch.setattr(cuda, "host_image", lambda h, w: np.empty((int(h), int(w), 4), np.float32))
    return lib


def test_the_renderer_satisfies_the_reference_protocols(ref_ol, stand_in):
    from ordinarylight.renderers.base import (ProductRendererProtocol, RendererImplementation, RendererProtocol,
                                              ResidentSceneRendererProtocol)
    from ordinarylight_b200 import CudaWavefrontRenderer

    r = CudaWavefrontRenderer(max_bounces=3)
    assert isinstance(r, RendererProtocol)
    assert isinstance(r, ProductRendererProtocol)
    assert isinstance(r, ResidentSceneRendererProtocol)
    info = type(r).implementation
    assert (info.name, info.family, info.graphics_api) == ("cuda-wavefront", "global_illumination", "cuda")
    assert isinstance(r, RendererImplementation) or hasattr(r, "implementation_info")
    r.close()
    r.close()


def test_the_reference_facade_drives_the_renderer(ref_ol, stand_in):
    from ordinarylight_b200 import CudaWavefrontRenderer, scenes
    from ordinarylight_b200.packing import pack_scene

    scene, camera = scenes.box_room(ref_ol)
    facade = ref_ol.Renderer(implementation=CudaWavefrontRenderer(max_bounces=4, samples_per_pixel=2))
    a = facade.render(scene, camera, (8, 6))
    b = facade.render(scene, camera, (8, 6))
    assert a.shape == (6, 8, 4) and a.dtype == np.float32
    assert float(a[0, 0, 0]) == 0.0 and float(b[0, 0, 0]) == 1.0
    facade.reset_sequence(5)
    c = facade.render(scene, camera, (8, 6))
    assert float(c[0, 0, 0]) == 5.0
    assert [f for *_rest, f in stand_in.renders] == [0, 1, 5]
    assert stand_in.resets == 1          # reset_sequence forgets the temporal history
    # one upload: the scene stays resident across frames of one revision
    packed = pack_scene(scene)
    assert stand_in.uploads == [dict(meshes=len(packed.mesh_vertex_offset) - 1, instances=len(packed.instance_mesh),
                                     materials=len(packed.materials), emitters=len(packed.emitters),
                                     lights=len(packed.lights), ref_volumes=0)]
    assert facade.last_timings["camera_rays"] == 8 * 6 * 2
    facade.close()


def test_the_reference_facade_passes_reference_volumes(ref_ol, stand_in):
    import parity_scenes
    from ordinarylight_b200 import CudaWavefrontRenderer

    scene, camera = parity_scenes.volume_room(ref_ol)
    facade = ref_ol.Renderer(implementation=CudaWavefrontRenderer(mode="reference_compatible", max_bounces=3))
    facade.render(scene, camera, (4, 4))
    assert stand_in.uploads[-1]["ref_volumes"] == 2
    facade.close()
