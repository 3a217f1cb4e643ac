"""Renderer facade: the reference's renderer-neutral API over an implementation.

Mirrors ``ordinarylight.Renderer`` (ordinarylight/renderer/_core.py:221-840)
for environments without the reference package, with the same sequencing
rules:

* calls run on one renderer-owned worker thread, in submission order
  (:263-265, :709-717);
* ``frame_index`` is reserved at submission and advances after every
  submission that did not pass one (:639-646);
* ``reset_sequence(k)`` is ordered behind queued jobs and resets the
  implementation's output history (:339-351, :447-451);
* returned colour is checked to be ``(height, width, 4) float32`` (:768-784).

``renderer_preference="cuda"`` constructs :class:`CudaWavefrontRenderer`;
with the reference installed, :func:`install_cuda_preference` adds the same
route to ``ordinarylight.Renderer``.
"""

from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass
from threading import Lock
from types import MappingProxyType

import numpy as np

_EXPECTED = {
    "color": (3, np.float32), "variance": (2, np.float32), "depth": (2, np.float32), "normal": (3, np.float32),
    "instance_id": (2, np.uint32), "object_id": (2, np.uint32), "material_id": (2, np.uint32),
    "motion": (3, np.float32),
}


class RenderStatistics(dict):
    """Measurements of one completed render (total_ms/gpu_ms aliases as in
    RenderStatistics, ordinarylight/renderer/_core.py:43-96)."""

    def __init__(self, *, frame_index, size, samples, timings):
        timings = dict(timings or {})
        super().__init__(frame_index=int(frame_index), width=int(size[0]), height=int(size[1]), samples=samples,
                         total_ms=timings.get("total_ms"), gpu_ms=timings.get("gpu_ms"))
        self.timings = MappingProxyType(timings)

    def __getattr__(self, name):
        try:
            return self[name]
        except KeyError as error:
            raise AttributeError(name) from error


@dataclass
class RenderJob:
    """Handle of an asynchronous render (RenderJob, renderer/_core.py:614-653)."""

    future: object
    frame_index: int

    def result(self, timeout=None):
        return self.future.result(timeout)

    def done(self):
        return self.future.done()

    def cancel(self):
        return self.future.cancel()


def _size(size):
    try:
        width, height = size
    except (TypeError, ValueError) as error:
        raise TypeError("size must be a (width, height) pair") from error
    width, height = int(width), int(height)
    if width <= 0 or height <= 0:
        raise ValueError("width and height must be positive")
    return width, height


class Renderer:
    """Render scenes to HDR arrays through a RendererProtocol implementation."""

    def __init__(self, *, config=None, implementation=None, renderer_preference="auto", **config_options):
        if config is not None and config_options:
            raise TypeError("pass config or renderer options, not both")
        if implementation is not None and (config is not None or config_options):
            raise TypeError("a supplied implementation owns its configuration")
        if implementation is not None and renderer_preference != "auto":
            raise TypeError("renderer_preference cannot be used with a supplied implementation")
        if implementation is None:
            if renderer_preference not in ("auto", "gi", "cuda"):
                raise ValueError("renderer_preference must be 'auto', 'gi' or 'cuda' for this package")
            from .renderers.cuda import CudaRendererConfig, CudaWavefrontRenderer
            implementation = CudaWavefrontRenderer(config or CudaRendererConfig(**config_options))
        if not callable(getattr(implementation, "render_frame", None)):
            raise TypeError("implementation must implement RendererProtocol.render_frame()")
        if not callable(getattr(implementation, "close", None)):
            raise TypeError("implementation must provide close()")
        self._implementation = implementation
        self._frame_index = 0
        self._last_statistics = None
        self._state_lock = Lock()
        self._submission_lock = Lock()
        self._implementation_lock = Lock()
        self._accepting = True
        self._executor = ThreadPoolExecutor(max_workers=1, thread_name_prefix="ordinarylight-b200-render")

    @property
    def implementation(self):
        return self._implementation

    @property
    def config(self):
        return getattr(self._implementation, "config", None)

    @property
    def device(self):
        return getattr(self._implementation, "device", None)

    @property
    def last_timings(self):
        return dict(getattr(self._implementation, "last_timings", {}))

    @property
    def last_statistics(self):
        return self._last_statistics

    @property
    def frame_index(self):
        with self._state_lock:
            return self._frame_index

    @property
    def available_outputs(self):
        return tuple(getattr(self._implementation, "available_outputs", ("color",)))

    @property
    def capabilities(self):
        return getattr(self._implementation, "capabilities", {})

    def _check_open(self):
        if not self._accepting or self._implementation is None:
            raise RuntimeError("renderer is closed")

    def reset_sequence(self, frame_index=0):
        frame_index = int(frame_index)
        if frame_index < 0:
            raise ValueError("frame_index cannot be negative")
        with self._submission_lock:
            with self._state_lock:
                self._check_open()
                self._frame_index = frame_index
            self._executor.submit(self._reset_history).result()

    def _reset_history(self):
        with self._implementation_lock:
            reset = getattr(self._implementation, "reset_output_history", None)
            if callable(reset):
                reset()

    def replace_scene(self, scene, *, reset_sequence=True):
        with self._submission_lock:
            with self._state_lock:
                self._check_open()
            self._executor.submit(self._replace_scene, scene).result()
            if reset_sequence:
                with self._state_lock:
                    self._frame_index = 0
        return scene

    def _replace_scene(self, scene):
        with self._implementation_lock:
            replace = getattr(self._implementation, "replace_scene", None)
            if not callable(replace):
                raise RuntimeError("the active renderer implementation does not support resident scene replacement")
            replace(scene)
            self._last_statistics = None

    def reconfigure(self, **changes):
        if not changes:
            return self.config
        with self._submission_lock:
            with self._state_lock:
                self._check_open()
            return self._executor.submit(self._reconfigure, dict(changes)).result()

    def _reconfigure(self, changes):
        with self._implementation_lock:
            reconfigure = getattr(self._implementation, "reconfigure", None)
            if not callable(reconfigure):
                raise RuntimeError("the active renderer implementation requires renderer recreation for settings")
            config = reconfigure(**changes)
            self._last_statistics = None
            return config

    def render(self, scene, camera, size, *, samples=None, frame_index=None, out=None, outputs=None):
        return self.render_async(scene, camera, size, samples=samples, frame_index=frame_index, out=out,
                                 outputs=outputs).result()

    def render_async(self, scene, camera, size, *, samples=None, frame_index=None, out=None, outputs=None):
        width, height = _size(size)
        with self._submission_lock:
            with self._state_lock:
                self._check_open()
                current = self._frame_index if frame_index is None else int(frame_index)
                if current < 0:
                    raise ValueError("frame_index cannot be negative")
                self._frame_index = current + 1
            future = self._executor.submit(self._render_serialized, scene, camera, width, height, samples,
                                           current, out, outputs)
        return RenderJob(future, current)

    def _render_serialized(self, scene, camera, width, height, samples, current, out, outputs):
        with self._implementation_lock:
            named = outputs is not None
            requested = ("color",) if outputs is None else ((outputs,) if isinstance(outputs, str)
                                                            else tuple(outputs))
            unavailable = tuple(n for n in requested if n not in self.available_outputs)
            if unavailable:
                raise ValueError(f"unsupported render outputs {unavailable}; available outputs are "
                                 f"{self.available_outputs}")
            if not named and out is not None:
                if not isinstance(out, np.ndarray):
                    raise TypeError("out must be a NumPy array")
                if out.shape != (height, width, 4):
                    raise ValueError(f"out must have shape {(height, width, 4)}, got {out.shape}")
                if out.dtype != np.float32:
                    raise TypeError("out must use float32 components")
            if named and callable(getattr(self._implementation, "render_products", None)):
                products = self._implementation.render_products(scene, camera, width, height, outputs=requested,
                                                                samples=samples, frame_index=current)
            else:
                products = {"color": self._implementation.render_frame(scene, camera, width, height,
                                                                       samples=samples, frame_index=current)}
            for name in requested:
                value = np.asarray(products[name])
                ndim, dtype = _EXPECTED[name]
                shape = (height, width, 4) if name == "color" else (
                    (height, width, 3) if name == "normal" else (
                        (height, width, 2) if name == "motion" else (height, width)))
                if value.shape != shape or value.dtype != dtype:
                    raise RuntimeError(f"renderer returned invalid {name!r}; expected {np.dtype(dtype)} {shape}, "
                                       f"got {value.dtype} {value.shape}")
            self._last_statistics = RenderStatistics(frame_index=current, size=(width, height), samples=samples,
                                                     timings=self.last_timings)
            if named:
                return {name: products[name] for name in requested}
            color = products["color"]
            if out is not None:
                np.copyto(out, color)
                return out
            return color

    def close(self):
        with self._submission_lock:
            with self._state_lock:
                if not self._accepting:
                    return
                self._accepting = False
        self._executor.shutdown(wait=True, cancel_futures=True)
        with self._implementation_lock:
            if self._implementation is not None:
                self._implementation.close()
                self._implementation = None

    def __enter__(self):
        self._check_open()
        return self

    def __exit__(self, *_exc):
        self.close()


def install_cuda_preference(ordinarylight_module=None):
    """Add ``renderer_preference="cuda"`` to the reference's ``Renderer``.

    Wraps ``ordinarylight.renderer._core._default_implementation``
    (ordinarylight/renderer/_core.py:25-40) so ``"cuda"`` constructs a
    CudaWavefrontRenderer and every other preference keeps the reference's
    Vulkan selection.  Returns False when the reference is not importable.
    """
    try:
        import importlib

        core = importlib.import_module("ordinarylight.renderer._core")
    except ImportError:
        return False
    if getattr(core._default_implementation, "_cuda_route", False):
        return True
    original = core._default_implementation

    def _default_implementation(config, config_options, preference="auto"):
        if preference == "cuda":
            from .renderers.cuda import CudaRendererConfig, CudaWavefrontRenderer

            return CudaWavefrontRenderer(config or CudaRendererConfig(**config_options))
        return original(config, config_options, preference)

    _default_implementation._cuda_route = True
    core._default_implementation = _default_implementation
    return True


__all__ = ["Renderer", "RenderJob", "RenderStatistics", "install_cuda_preference"]
