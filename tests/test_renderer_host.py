"""The renderer facade (ordinarylight_b200/renderer.py) and the reference
hook (install_cuda_preference) on CPU, with a fake implementation in place
of the CUDA renderer, as the reference tests its facade with fakes
(types.SimpleNamespace and patched classes)."""
import sys
import types

import numpy as np
import pytest

from ordinarylight_b200.renderer import Renderer, install_cuda_preference


class FakeImplementation:
    """Records calls; returns an image whose value is the frame index."""

    available_outputs = ("color", "depth")

    def __init__(self, bad_shape=False):
        self.frames = []
        self.resets = 0
        self.closed = 0
        self.bad_shape = bad_shape
        self.last_timings = {"total_ms": 1.5, "gpu_ms": 1.0}

    def render_frame(self, scene, camera, width, height, *, samples=None, frame_index=0):
        self.frames.append(frame_index)
        h = height + 1 if self.bad_shape else height
        return np.full((h, width, 4), float(frame_index), np.float32)

    def render_products(self, scene, camera, width, height, *, outputs, samples=None, frame_index=0):
        self.frames.append(frame_index)
        out = {"color": np.zeros((height, width, 4), np.float32), "depth": np.ones((height, width), np.float32)}
        return {name: out[name] for name in outputs}

    def reset_output_history(self):
        self.resets += 1

    def close(self):
        self.closed += 1


def test_frame_indices_advance_per_submission_and_reset_in_order():
    impl = FakeImplementation()
    r = Renderer(implementation=impl)
    a = r.render(None, None, (4, 3))
    b = r.render(None, None, (4, 3))
    assert a.shape == (3, 4, 4) and a.dtype == np.float32
    assert float(a[0, 0, 0]) == 0.0 and float(b[0, 0, 0]) == 1.0
    job = r.render_async(None, None, (4, 3), frame_index=7)
    assert job.frame_index == 7 and float(job.result()[0, 0, 0]) == 7.0
    assert r.frame_index == 8
    r.reset_sequence(3)
    assert impl.resets == 1 and r.frame_index == 3
    r.render(None, None, (4, 3))
    assert impl.frames == [0, 1, 7, 3]
    stats = r.last_statistics
    assert stats.frame_index == 3 and stats.width == 4 and stats.height == 3 and stats.total_ms == 1.5
    with pytest.raises(ValueError):
        r.reset_sequence(-1)
    r.close()


def test_out_buffer_is_validated_and_filled():
    r = Renderer(implementation=FakeImplementation())
    out = np.empty((3, 4, 4), np.float32)
    assert r.render(None, None, (4, 3), out=out, frame_index=5) is out
    assert np.all(out == 5.0)
    with pytest.raises(ValueError):
        r.render(None, None, (4, 3), out=np.empty((4, 4, 4), np.float32))
    with pytest.raises(TypeError):
        r.render(None, None, (4, 3), out=np.empty((3, 4, 4), np.float64))
    with pytest.raises(ValueError):
        r.render(None, None, (0, 3))
    with pytest.raises(TypeError):
        r.render(None, None, 12)
    r.close()


def test_named_outputs_and_contract_violations():
    r = Renderer(implementation=FakeImplementation())
    products = r.render(None, None, (4, 3), outputs=("color", "depth"))
    assert set(products) == {"color", "depth"} and products["depth"].shape == (3, 4)
    with pytest.raises(ValueError):
        r.render(None, None, (4, 3), outputs=("normal",))
    r.close()
    bad = Renderer(implementation=FakeImplementation(bad_shape=True))
    with pytest.raises(RuntimeError):
        bad.render(None, None, (4, 3))
    bad.close()


def test_close_is_idempotent_and_later_calls_raise():
    impl = FakeImplementation()
    r = Renderer(implementation=impl)
    r.close()
    r.close()
    assert impl.closed == 1
    with pytest.raises(RuntimeError):
        r.render(None, None, (4, 3))
    with pytest.raises(RuntimeError):
        r.reset_sequence(0)


def test_constructor_rejects_conflicting_arguments():
    with pytest.raises(TypeError):
        Renderer(implementation=FakeImplementation(), renderer_preference="cuda")
    with pytest.raises(TypeError):
        Renderer(implementation=FakeImplementation(), max_bounces=4)
    with pytest.raises(TypeError):
        Renderer(config=object(), max_bounces=4)
    with pytest.raises(ValueError):
        Renderer(renderer_preference="vulkan")
    with pytest.raises(TypeError):
        Renderer(implementation=types.SimpleNamespace(close=lambda: None))


def test_cuda_implementation_identity_without_a_device():
    from ordinarylight_b200.renderers.base import RendererImplementation
    from ordinarylight_b200.renderers.cuda import CudaWavefrontRenderer

    assert issubclass(CudaWavefrontRenderer, RendererImplementation)
    info = CudaWavefrontRenderer.implementation_info()
    assert info.name == "cuda-wavefront" and info.family == "global_illumination"
    assert "color" in CudaWavefrontRenderer.available_outputs


def test_install_cuda_preference_routes_cuda_and_keeps_the_rest(monkeypatch):
    calls = []

    def original(config, config_options, preference="auto"):
        calls.append(preference)
        return ("vulkan", preference)

    core = types.ModuleType("ordinarylight.renderer._core")
    core._default_implementation = original
    package = types.ModuleType("ordinarylight")
    package.__path__ = []
    sub = types.ModuleType("ordinarylight.renderer")
    sub.__path__ = []
    sub._core = core
    package.renderer = sub
    monkeypatch.setitem(sys.modules, "ordinarylight", package)
    monkeypatch.setitem(sys.modules, "ordinarylight.renderer", sub)
    monkeypatch.setitem(sys.modules, "ordinarylight.renderer._core", core)

    from ordinarylight_b200.renderers import cuda

    class StubCuda:
        def __init__(self, config):
            self.config = config

    monkeypatch.setattr(cuda, "CudaWavefrontRenderer", StubCuda)
    assert install_cuda_preference() is True
    assert install_cuda_preference() is True            # a second install keeps one wrapper
    routed = core._default_implementation
    assert routed._cuda_route
    made = routed(None, {"max_bounces": 3}, "cuda")
    assert isinstance(made, StubCuda) and made.config.max_bounces == 3
    assert routed(None, {}, "auto") == ("vulkan", "auto") and calls == ["auto"]


def test_install_cuda_preference_without_the_reference(monkeypatch):
    monkeypatch.setitem(sys.modules, "ordinarylight.renderer._core", None)
    assert install_cuda_preference() is False
