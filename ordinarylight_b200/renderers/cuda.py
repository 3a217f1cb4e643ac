"""``renderers.cuda``: the B200 wavefront path tracer behind RendererProtocol.

A drop-in ``RendererImplementation`` for OrdinaryLight's renderer facade:
``ol.Renderer(implementation=CudaWavefrontRenderer(...))`` (or the
``renderer_preference="cuda"`` route of :func:`ordinarylight_b200.Renderer`)
renders ``(height, width, 4)`` float32 linear HDR through hand-written sm_100a
kernels in ``libolcuda.so``.  It replaces the Vulkan GI engine's offscreen
path (``_VulkanGlobalIlluminationEngine.render_frame`` ->
``render_wavefront_outputs``, ordinarylight/targets/vulkan/api.py:1233-1451)
and matches the contract of ``CpuReferenceRenderer``
(ordinarylight/renderers/reference/cpu.py:24-75):

* ``render_frame(scene, camera, w, h, *, samples=None, frame_index=0)``;
  the seed of a frame is ``config.seed + frame_index`` and identical
  (scene, camera, size, samples, frame_index) give identical bytes;
* ``ValueError`` for invalid sizes and sample counts, ``RuntimeError`` after
  ``close()`` (which is idempotent);
* ``last_timings`` with ``total_ms``/``gpu_ms`` (read by RenderStatistics,
  ordinarylight/renderer/_core.py:43-96) plus ray counts and Mrays/s.

``mode="reference_compatible"`` reproduces the CPU reference's estimator
(Lambert, emission on every hit, CPU sky, no NEE) for parity; the default
``mode="production"`` is the GPU wavefront's GGX/Lambert transport with
next-event estimation, MIS, Russian roulette and optional ReSTIR DI.
"""

from __future__ import annotations

from collections import OrderedDict
from dataclasses import asdict, dataclass, fields, replace
import ctypes
import time

import numpy as np

from .. import _native
from ..packing import PackedScene, refit_mask, pack_camera, pack_scene
from .base import RendererImplementation, RendererImplementationInfo

_MODES = {"production": _native.MODE_PRODUCTION, "reference_compatible": _native.MODE_REFERENCE_COMPATIBLE}
_PRODUCTS = ("color", "variance", "depth", "normal", "instance_id", "object_id", "material_id", "motion")


@dataclass(frozen=True)
class CudaRendererConfig:
    """Frozen renderer configuration: ReferenceConfig's fields
    (cpu.py:9-21) plus the wavefront knobs."""

    samples_per_pixel: int = 1
    max_bounces: int = 3
    seed: int = 1
    mode: str = "production"
    device: int = 0
    russian_roulette_start: int = 3
    russian_roulette_min_survival: float = 0.1
    restir: bool = False
    restir_candidates: int = 32
    restir_temporal: bool = True
    restir_spatial: int = 1
    restir_neighbours: int = 5
    restir_radius: float = 30.0
    restir_max_history: int = 20
    block_size: int = 256
    trace_block: int = 128
    stack_depth: int = 24
    chunk_paths: int = 0
    use_graphs: bool = True
    flatten_instances: bool = True
    trace_scheduler: str = "refill"
    nee: bool = True
    sort_rays: bool = False
    serve_aging_steps: int = 8
    sample_variance: bool = False
    denoiser_signal_capture: bool = False

    def __post_init__(self):
        if not 1 <= int(self.samples_per_pixel) <= 65536:
            raise ValueError("samples_per_pixel must be between 1 and 65536")
        if not 1 <= int(self.max_bounces) <= 64:
            raise ValueError("max_bounces must be between 1 and 64")
        if int(self.seed) < 0:
            raise ValueError("seed cannot be negative")
        if self.mode not in _MODES:
            raise ValueError(f"mode must be one of {tuple(_MODES)}")
        if int(self.device) < 0:
            raise ValueError("device cannot be negative")
        if not 0 <= int(self.russian_roulette_start) <= 64:
            raise ValueError("russian_roulette_start must be between 0 and 64")
        if not 0.0 <= float(self.russian_roulette_min_survival) <= 1.0:
            raise ValueError("russian_roulette_min_survival must be between 0 and 1")
        if not 1 <= int(self.restir_candidates) <= 64:
            raise ValueError("restir_candidates must be between 1 and 64")
        if not 0 <= int(self.restir_spatial) <= 4:
            raise ValueError("restir_spatial must be between 0 and 4")
        if not 0 <= int(self.restir_neighbours) <= 16:
            raise ValueError("restir_neighbours must be between 0 and 16")
        if not float(self.restir_radius) > 0.0:
            raise ValueError("restir_radius must be positive")
        if int(self.stack_depth) not in (16, 24, 32):
            raise ValueError("stack_depth must be 16, 24 or 32")
        if int(self.block_size) % 32 or not 64 <= int(self.block_size) <= 1024:
            raise ValueError("block_size must be a multiple of 32 in [64, 1024]")
        if int(self.trace_block) not in (64, 128, 256):
            raise ValueError("trace_block must be 64, 128 or 256")
        if int(self.chunk_paths) < 0:
            raise ValueError("chunk_paths cannot be negative")
        if self.trace_scheduler not in ("refill", "batch"):
            raise ValueError("trace_scheduler must be 'refill' or 'batch'")

    def native(self) -> _native.OlcConfig:
        c = _native.OlcConfig()
        c.device = int(self.device)
        c.mode = _MODES[self.mode]
        c.max_bounces = int(self.max_bounces)
        c.seed = int(self.seed) & 0xFFFFFFFF
        c.russian_roulette_start = int(self.russian_roulette_start)
        c.russian_roulette_min_survival = float(self.russian_roulette_min_survival)
        c.restir = int(bool(self.restir))
        c.restir_candidates = int(self.restir_candidates)
        c.restir_temporal = int(bool(self.restir_temporal))
        c.restir_spatial = int(self.restir_spatial)
        c.restir_neighbours = int(self.restir_neighbours)
        c.restir_radius = float(self.restir_radius)
        c.restir_max_history = int(self.restir_max_history)
        c.block_size = int(self.block_size)
        c.trace_block = int(self.trace_block)
        c.stack_depth = int(self.stack_depth)
        c.chunk_paths = int(self.chunk_paths)
        c.use_graphs = int(bool(self.use_graphs))
        c.flatten_instances = int(bool(self.flatten_instances))
        c.trace_scheduler = 0 if self.trace_scheduler == "refill" else 1
        c.disable_nee = 0 if self.nee else 1
        c.ray_sort = 1 if self.sort_rays else 0
        c.serve_aging_steps = int(self.serve_aging_steps)
        c.sample_variance = 1 if self.sample_variance else 0
        return c


@dataclass(frozen=True)
class RenderRequest:
    """One render job of a batch or of a served stream: what
    ``Renderer.render_async`` (ordinarylight/renderer/_core.py:614-651)
    submits, plus a per-job bounce limit.  ``samples=None`` and
    ``max_bounces=None`` take the renderer configuration's values."""

    scene: object
    camera: object
    width: int
    height: int
    samples: int | None = None
    frame_index: int = 0
    max_bounces: int | None = None
    first_sample: int = 0       # RNG index of the first sample (a shard of a frame's samples)


def _packed(scene, mode: str) -> PackedScene:
    """The arrays of a scene: a reference or mirror ``Scene`` is flattened;
    an already packed scene (``PackedScene``, for instance one loaded from a
    file written where the scene objects exist) is used as it is.  The
    production transport's medium is one density grid: a scene with several
    visible volumes renders only in the reference-compatible mode, whose ray
    march integrates up to eight."""
    packed = scene if isinstance(scene, PackedScene) else pack_scene(scene)
    if mode == "production" and packed.volume_count > 1:
        raise RuntimeError("the production transport supports one visible volume per scene")
    return packed


def host_image(height: int, width: int) -> np.ndarray:
    """(height, width, 4) float32 host array in page-locked memory (torch's
    caching host allocator), so the device-to-host copy of a frame runs at
    full link bandwidth instead of through a pageable bounce buffer.  The
    array returns to the allocator's cache when it is dropped."""
    import torch

    return torch.empty((int(height), int(width), 4), dtype=torch.float32, pin_memory=True).numpy()


class CudaWavefrontRenderer(RendererImplementation):
    """Wavefront path tracer on one CUDA device (sm_100a kernels)."""

    available_outputs = _PRODUCTS
    implementation = RendererImplementationInfo(name="cuda-wavefront", family="global_illumination",
                                                graphics_api="cuda")

    def __init__(self, config: CudaRendererConfig | None = None, **options):
        if config is not None and options:
            raise TypeError("pass config or renderer options, not both")
        self.config = config or CudaRendererConfig(**options)
        if not isinstance(self.config, CudaRendererConfig):
            raise TypeError("config must be a CudaRendererConfig")
        self._lib = _native.load()
        handle = ctypes.c_void_p()
        _native.check(self._lib, None, self._lib.olc_create(ctypes.byref(self.config.native()),
                                                             ctypes.byref(handle)))
        self._ctx = handle
        self._closed = False
        self._scene_key = None
        self._packed = None
        self._scene_obj = None
        self.last_update = None          # what the last in-place scene update did
        self._resident_packed = {}       # pool handle -> PackedScene it holds
        self._output_history = None      # previous products frame of the motion output
        self._resident = OrderedDict()   # (id(scene), revision) -> (handle, scene)
        self._served_outputs = {}        # ticket -> output array
        self.last_timings = {}
        self.device = f"cuda:{self.config.device}"

    # -- identity / capabilities --------------------------------------------
    @property
    def capabilities(self):
        return {
            "renderer": "cuda-wavefront",
            "outputs": self.available_outputs,
            "features": frozenset({"offscreen_rendering", "instancing", "next_event_estimation",
                                   "restir_di", "deterministic_sequences", "resident_scenes"}),
            "limits": {"max_bounces": 64, "max_samples_per_pixel": 65536},
            "device": self.device,
        }

    def _require_open(self):
        if self._closed:
            raise RuntimeError("cuda renderer is closed")

    # -- scene residency -------------------------------------------------------
    def _ensure_scene(self, scene, force=False):
        key = (id(scene), getattr(scene, "revision", None))
        if not force and key == self._scene_key:
            return 0.0
        t0 = time.perf_counter()
        packed = _packed(scene, self.config.mode)
        self.last_update = None
        if (not force and self._packed is not None and self._scene_obj is scene
                and self._update_in_place(_native.DEFAULT_SCENE, self._packed, packed)):
            pass
        else:
            desc = packed.descriptor()
            _native.check(self._lib, self._ctx, self._lib.olc_upload_scene(self._ctx, ctypes.byref(desc)))
        self._packed = packed
        self._scene_obj = scene
        self._scene_key = key
        return (time.perf_counter() - t0) * 1e3

    def _update_in_place(self, handle, old, new) -> bool:
        """Refit/rewrite a resident scene for ``new`` when the reference's
        in-place update rules allow it (see :func:`packing.refit_mask`)."""
        mask = refit_mask(old, new)
        if mask is None:
            return False
        desc = new.descriptor()
        applied, refitted = ctypes.c_int32(), ctypes.c_uint32()
        _native.check(self._lib, self._ctx, self._lib.olc_update_scene(
            self._ctx, handle, ctypes.byref(desc), _native.ptr(mask) if len(mask) else None,
            ctypes.byref(applied), ctypes.byref(refitted)))
        if not applied.value:
            return False
        self.last_update = {"refitted_blas": int(refitted.value), "meshes": int(len(mask))}
        return True

    def replace_scene(self, scene) -> None:
        """Make ``scene`` resident (ResidentSceneRendererProtocol,
        ordinarylight/renderers/base.py:106-112).  On failure the previous
        scene stays resident."""
        self._require_open()
        self._ensure_scene(scene, force=True)
        self.reset_output_history()

    def scene_bytes(self) -> int:
        value = ctypes.c_uint64()
        _native.check(self._lib, self._ctx, self._lib.olc_scene_bytes(self._ctx, ctypes.byref(value)))
        return int(value.value)

    # -- rendering -----------------------------------------------------------
    def _render(self, scene, camera, width, height, samples, frame_index, out_ptr, out_is_device):
        width, height = int(width), int(height)
        if width <= 0 or height <= 0:
            raise ValueError("width and height must be positive")
        spp = self.config.samples_per_pixel if samples is None else int(samples)
        if not 1 <= spp <= 65536:
            raise ValueError("samples must be between 1 and 65536")
        frame_index = int(frame_index)
        if frame_index < 0:
            raise ValueError("frame_index cannot be negative")
        t0 = time.perf_counter()
        upload_ms = self._ensure_scene(scene)
        cam = pack_camera(camera)
        stats = _native.OlcRenderStats()
        status = self._lib.olc_render(self._ctx, ctypes.byref(cam), width, height, spp, frame_index & 0xFFFFFFFF,
                                      out_ptr, int(out_is_device), ctypes.byref(stats))
        _native.check(self._lib, self._ctx, status)
        total_ms = (time.perf_counter() - t0) * 1e3
        rays = stats.camera_rays + stats.extension_rays + stats.shadow_rays
        gpu_ms = float(stats.gpu_ms)
        self.last_timings = {
            "total_ms": total_ms,
            "gpu_ms": gpu_ms,
            "scene_upload_ms": upload_ms,
            "camera_rays": int(stats.camera_rays),
            "extension_rays": int(stats.extension_rays),
            "shadow_rays": int(stats.shadow_rays),
            "rays": int(rays),
            "closest_hit_rays": int(stats.camera_rays + stats.extension_rays),
            "mrays_per_s": rays / (gpu_ms * 1e3) if gpu_ms > 0 else 0.0,
            "queue_overflow": int(stats.overflow),
            "traversal_errors": int(stats.traversal_errors),
            "chunks": int(stats.chunks),
            "restir_history_used": bool(stats.restir_history_used),
            "samples_per_pixel": spp,
            "h2d_bytes": int(stats.h2d_bytes),
            "d2h_bytes": int(stats.d2h_bytes),
        }
        if stats.traversal_errors:
            raise RuntimeError(f"{stats.traversal_errors} traversal stack overflows")

    def render_frame(self, scene, camera, width, height, *, samples=None, frame_index=0):
        """Render one linear-HDR frame as a (height, width, 4) float32 array."""
        self._require_open()
        width, height = int(width), int(height)
        if width <= 0 or height <= 0:
            raise ValueError("width and height must be positive")
        out = host_image(height, width)
        self._render(scene, camera, width, height, samples, frame_index, _native.ptr(out), False)
        return out

    render_wavefront = render_frame

    def render_frame_into(self, scene, camera, width, height, out, *, samples=None, frame_index=0):
        """Render into a caller-owned buffer: a host numpy array or a device
        tensor (anything with ``data_ptr()``) of height*width*4 float32."""
        self._require_open()
        on_device = hasattr(out, "data_ptr") and getattr(out, "is_cuda", False)
        if hasattr(out, "numel"):
            count = out.numel()
        else:
            count = out.size
            if out.dtype != np.float32 or not out.flags.c_contiguous:
                raise TypeError("out must be a contiguous float32 array")
        if count != int(width) * int(height) * 4:
            raise ValueError("out must hold height*width*4 float32 values")
        self._render(scene, camera, width, height, samples, frame_index, _native.ptr(out), on_device)
        return out

    def render_products(self, scene, camera, width, height, *, outputs, samples=None, frame_index=0):
        """Named products (ProductRendererProtocol, base.py:74-90): ``color``,
        the per-pixel luminance ``variance`` over the frame's samples
        (api.py:1400-1433), and the first sample's primary-hit ``depth``,
        ``normal``, ``instance_id``/``object_id`` and ``material_id`` (shapes
        of ordinarylight/renderer/_core.py:768-777).  Asking for ``variance``
        switches ``sample_variance`` on for this and later frames."""
        self._require_open()
        requested = (outputs,) if isinstance(outputs, str) else tuple(outputs)
        unknown = [name for name in requested if name not in self.available_outputs]
        if unknown:
            raise ValueError(f"unsupported render outputs {tuple(unknown)}")
        if "variance" in requested and not self.config.sample_variance:
            self.reconfigure(sample_variance=True)
        color = self.render_frame(scene, camera, width, height, samples=samples, frame_index=frame_index)
        h, w = int(height), int(width)
        variance = None
        if "variance" in requested:
            variance = np.empty((h, w), np.float32)
            _native.check(self._lib, self._ctx, self._lib.olc_read_variance(self._ctx, w, h, _native.ptr(variance), 0))
        depth = np.empty((h, w), np.float32)
        normal = np.empty((h, w, 3), np.float32)
        inst = np.empty((h, w), np.uint32)
        mat = np.empty((h, w), np.uint32)
        _native.check(self._lib, self._ctx, self._lib.olc_read_products(
            self._ctx, w, h, _native.ptr(depth), _native.ptr(normal), _native.ptr(inst), _native.ptr(mat), None))
        table = {"color": color, "variance": variance, "depth": depth, "normal": normal, "instance_id": inst,
                 "object_id": inst.copy(), "material_id": mat}
        if "motion" in requested:
            table["motion"] = self._motion_product(scene, camera, w, h)
            self._capture_motion_state(scene, camera, (w, h))
        return {name: table[name] for name in requested}

    def sample_texture(self, scene, binding, uv0, uv1, footprint0, footprint1, *, srgb):
        """The shading stage's lookup of texture binding ``binding`` of
        ``scene`` at n points (its parity tests): (n, 4) float32."""
        self._require_open()
        self._ensure_scene(scene)
        uv0 = np.ascontiguousarray(uv0, np.float32)
        uv1 = np.ascontiguousarray(uv1, np.float32)
        fp0 = np.ascontiguousarray(footprint0, np.float32)
        fp1 = np.ascontiguousarray(footprint1, np.float32)
        out = np.empty((len(uv0), 4), np.float32)
        _native.check(self._lib, self._ctx, self._lib.olc_sample_texture(
            self._ctx, _native.DEFAULT_SCENE, int(binding), len(uv0), _native.ptr(uv0), _native.ptr(uv1),
            _native.ptr(fp0), _native.ptr(fp1), 1 if srgb else 0, _native.ptr(out)))
        return out

    # -- denoiser inputs ----------------------------------------------------------
    def capture_denoiser_raw(self, scene, camera, width, height, *, frame_index=0):
        """One-sample frame and its denoiser path signals
        (capture_denoiser_raw, ordinarylight/targets/vulkan/api.py:1453-1582):
        the radiance is split between a diffuse and a specular channel by the
        primary material's specular-lobe probability, as the reference's
        path-to-HDR partition does (not physically separated lobes), and both
        carry the distance from the primary hit to the path's next surface
        vertex (0 when it has none).  Needs ``denoiser_signal_capture=True``."""
        self._require_open()
        if not self.config.denoiser_signal_capture:
            raise RuntimeError("capture_denoiser_raw requires denoiser_signal_capture=True")
        width, height = int(width), int(height)
        if width < 1 or height < 1:
            raise ValueError("width and height must be positive")
        radiance = self.render_frame(scene, camera, width, height, samples=1, frame_index=frame_index)
        depth = np.empty((height, width), np.float32)
        normal = np.empty((height, width, 3), np.float32)
        prim = np.empty((height, width), np.uint32)
        _native.check(self._lib, self._ctx, self._lib.olc_read_products(
            self._ctx, width, height, _native.ptr(depth), _native.ptr(normal), None, None, _native.ptr(prim)))
        position, bary = self.hit_geometry(width, height)
        signals = np.empty((height, width, 4), np.float32)
        secondary = np.empty((height, width, 4), np.float32)
        _native.check(self._lib, self._ctx, self._lib.olc_read_path_signals(
            self._ctx, width, height, _native.ptr(signals), _native.ptr(secondary)))
        resolved = np.maximum(radiance[..., :3], 0.0)
        captured = signals[..., 1] > 0.5
        probability = np.where(captured, np.clip(signals[..., 0], 0.0, 1.0), 0.0)[..., None].astype(np.float32)
        distance = np.zeros((height, width), np.float32)
        valid = captured & (secondary[..., 3] > 0.5)
        distance[valid] = np.linalg.norm(secondary[valid, :3] - position[valid], axis=-1)
        diffuse = np.empty((height, width, 4), np.float32)
        specular = np.empty((height, width, 4), np.float32)
        diffuse[..., :3] = resolved * (1.0 - probability)
        specular[..., :3] = resolved * probability
        diffuse[..., 3] = distance
        specular[..., 3] = distance
        path_state = {"diffuse_radiance_hit_distance": diffuse, "specular_radiance_hit_distance": specular,
                      "specular_probability": probability[..., 0], "secondary_position": secondary}
        return {"radiance": radiance, "path_state": path_state, "depth": depth, "normal": normal,
                "primitive_id": prim, "primary_position": position, "primary_barycentric": bary}

    def capture_denoiser_signals(self, scene, camera, width, height, *, frame_index=0):
        """Canonical diffuse/specular denoiser inputs of one frame
        (capture_denoiser_signals, ordinarylight/targets/vulkan/api.py:1584-1660):
        radiance and hit distance per channel, unit normal and material
        roughness, linear view depth, motion from the pixel centre to its
        previous-frame location, material ids, and the frame's matrices."""
        try:
            from ordinarylight.denoising import DenoiserFrameInfo, DenoiserSignals
        except ImportError:
            from ..denoising import DenoiserFrameInfo, DenoiserSignals
        from ..denoising import camera_matrix

        raw = self.capture_denoiser_raw(scene, camera, width, height, frame_index=frame_index)
        width, height = int(width), int(height)
        prim = raw["primitive_id"]
        foreground = prim != np.uint32(0xFFFFFFFF)
        material_id = np.full((height, width), np.uint32(0xFFFFFFFF), np.uint32)
        ids = np.empty((height, width), np.uint32)
        _native.check(self._lib, self._ctx, self._lib.olc_read_products(
            self._ctx, width, height, None, None, None, _native.ptr(ids), None))
        material_id[foreground] = ids[foreground]
        normal_roughness = np.zeros((height, width, 4), np.float32)
        normal_roughness[..., :3] = raw["normal"]
        lengths = np.linalg.norm(normal_roughness[..., :3], axis=-1)
        ok = foreground & (lengths > 1e-12)
        normal_roughness[ok, :3] /= lengths[ok, None]
        material_id_of = getattr(scene, "material_id", None)
        meshes = getattr(scene, "render_meshes", None) or scene.visible_meshes
        for mesh in meshes:
            if callable(material_id_of):
                normal_roughness[material_id == material_id_of(mesh.material), 3] = float(mesh.material.roughness)
        origin = np.asarray(camera.position, np.float64)
        forward = np.asarray(camera.target, np.float64) - origin
        forward /= np.linalg.norm(forward)
        view_z = np.zeros((height, width), np.float32)
        view_z[foreground] = ((raw["primary_position"][foreground] - origin) @ forward).astype(np.float32)
        previous = self._output_history
        compatible = previous is not None and previous["scene"] is scene and previous["size"] == (width, height)
        motion = self._motion_product(scene, camera, width, height)
        if compatible:
            # previous-minus-current from the pixel centre, including the
            # current ray jitter (api.py:1630-1641)
            now = self._motion_camera(camera)
            o = np.asarray(now.origin[:], np.float64)
            f, r_, u = (np.asarray(getattr(now, k)[:], np.float64) for k in ("forward", "right", "up"))
            rel = raw["primary_position"].reshape(-1, 3).astype(np.float64) - o
            dist = rel @ f
            safe = np.maximum(dist, 1e-12)
            px = ((rel @ r_) / (safe * now.scale * (width / height)) + 1.0) * 0.5 * width
            py = (-(rel @ u) / (safe * now.scale) + 1.0) * 0.5 * height
            yy, xx = np.indices((height, width))
            projected = np.stack((px.reshape(height, width), py.reshape(height, width)), axis=-1)
            centres = np.stack((xx, yy), axis=-1) + 0.5
            motion = (projected - centres - motion).astype(np.float32)
            motion[~(foreground & (dist.reshape(height, width) > 1e-8))] = 0.0
        current = camera_matrix(camera, width, height)
        before = camera_matrix(previous["camera"], width, height) if compatible else current
        self._capture_motion_state(scene, camera, (width, height))
        ps = raw["path_state"]
        return DenoiserSignals(
            np.ascontiguousarray(ps["diffuse_radiance_hit_distance"], np.float32),
            np.ascontiguousarray(ps["specular_radiance_hit_distance"], np.float32),
            normal_roughness, view_z, motion, material_id,
            DenoiserFrameInfo(current, before, int(frame_index), camera_cut=not compatible))

    def hit_geometry(self, width, height):
        """World hit points (h, w, 3) and barycentrics (h, w, 2) of the last
        render's first-sample primary hits."""
        pos = np.empty((int(height), int(width), 3), np.float32)
        bary = np.empty((int(height), int(width), 2), np.float32)
        _native.check(self._lib, self._ctx, self._lib.olc_read_hit_geometry(
            self._ctx, int(width), int(height), _native.ptr(pos), _native.ptr(bary)))
        return pos, bary

    @staticmethod
    def _motion_camera(camera):
        """_project_positions' frame (api.py:1118-1136) in double precision."""
        origin = np.asarray(camera.position, np.float64)
        forward = np.asarray(camera.target, np.float64) - origin
        forward /= np.linalg.norm(forward)
        right = np.cross(forward, np.asarray(camera.up, np.float64))
        right /= np.linalg.norm(right)
        up = np.cross(right, forward)
        c = _native.OlcMotionCamera()
        for name, v in (("origin", origin), ("forward", forward), ("right", right), ("up", up)):
            getattr(c, name)[:] = [float(x) for x in v]
        c.scale = float(np.tan(np.radians(camera.vertical_fov_degrees) * 0.5))
        return c

    def _motion_product(self, scene, camera, width, height):
        """Screen-space motion of the first sample's primary hits since the
        previous motion frame (_motion_product, api.py:1151-1200): meshes
        match by Mesh.id and need the same topology and vertex count."""
        motion = np.zeros((height, width, 2), np.float32)
        previous = self._output_history
        if previous is None or previous["scene"] is not scene or previous["size"] != (width, height):
            return motion
        table, offset = [], 0
        for mesh in scene.visible_meshes:
            count = len(mesh.indices)
            old = previous["meshes"].get(mesh.id)
            first = 0xFFFFFFFF
            if count and old is not None:
                old_indices, old_vertex_count, old_first = old
                if (old_indices.shape == mesh.indices.shape and np.array_equal(old_indices, mesh.indices)
                        and old_vertex_count == len(mesh.vertices)):
                    first = old_first
            if count:
                table.append((offset, count, first))
            offset += count
        meshes = (_native.OlcMotionMesh * max(len(table), 1))()
        for k, (first, count, prev) in enumerate(table):
            meshes[k].first, meshes[k].count, meshes[k].previous_first = first, count, prev
        now, before = self._motion_camera(camera), self._motion_camera(previous["camera"])
        _native.check(self._lib, self._ctx, self._lib.olc_read_motion(
            self._ctx, width, height, meshes, len(table), ctypes.byref(now), ctypes.byref(before),
            _native.ptr(motion)))
        return motion

    def _capture_motion_state(self, scene, camera, size):
        """Keep this frame as the motion history (_capture_motion_state,
        api.py:1139-1149): topology per Mesh.id on the host, world-space
        triangles on the device."""
        meshes, offset = {}, 0
        for mesh in scene.visible_meshes:
            meshes[mesh.id] = (np.array(mesh.indices, copy=True), len(mesh.vertices), offset)
            offset += len(mesh.indices)
        _native.check(self._lib, self._ctx, self._lib.olc_capture_motion_state(self._ctx))
        self._output_history = {"scene": scene, "camera": camera, "size": size, "meshes": meshes}

    def primitive_ids(self, width, height):
        """Packed primitive index of the last render's first-sample primary hits."""
        prim = np.empty((int(height), int(width)), np.uint32)
        _native.check(self._lib, self._ctx, self._lib.olc_read_products(
            self._ctx, int(width), int(height), None, None, None, None, _native.ptr(prim)))
        return prim

    # -- resident scene pool ---------------------------------------------------
    def resident_scene(self, scene) -> int:
        """Handle of ``scene`` in the device scene pool, uploading it on first
        use.  Keyed by (scene object, ``Scene.revision``) like the reference's
        resident scene (ordinarylight/targets/vulkan/core.py:4591-4611)."""
        self._require_open()
        key = (id(scene), getattr(scene, "revision", None))
        entry = self._resident.get(key)
        if entry is not None:
            self._resident.move_to_end(key)
            return entry[0]
        packed = _packed(scene, self.config.mode)
        self.last_update = None
        # an older revision of the same scene is updated in place when the
        # in-place rules allow it and no queued job still renders it
        stale = [k for k, (_h, sc) in self._resident.items() if sc is scene]
        for old_key in stale:
            handle = self._resident[old_key][0]
            try:
                updated = self._update_in_place(handle, self._resident_packed[handle], packed)
            except RuntimeError:
                updated = False
            if updated:
                del self._resident[old_key]
                self._resident[key] = (handle, scene)
                self._resident_packed[handle] = packed
                return handle
        desc = packed.descriptor()
        handle = ctypes.c_uint32()
        _native.check(self._lib, self._ctx, self._lib.olc_add_scene(self._ctx, ctypes.byref(desc),
                                                                    ctypes.byref(handle)))
        # the entry keeps the scene alive so that its id() is not reused
        self._resident[key] = (int(handle.value), scene)
        self._resident_packed[int(handle.value)] = packed
        return int(handle.value)

    def release_scene(self, scene) -> None:
        """Drop ``scene`` from the pool (its ranges are reused)."""
        self._require_open()
        key = (id(scene), getattr(scene, "revision", None))
        entry = self._resident.pop(key, None)
        if entry is None:
            raise ValueError("scene is not resident")
        self._resident_packed.pop(entry[0], None)
        _native.check(self._lib, self._ctx, self._lib.olc_remove_scene(self._ctx, entry[0]))

    def resident_scenes(self):
        """Resident pool scenes in least-recently-used order: (scene, handle, bytes)."""
        out = []
        for handle, scene in self._resident.values():
            stats = _native.OlcSceneStats()
            _native.check(self._lib, self._ctx, self._lib.olc_scene_stats_get(self._ctx, handle,
                                                                              ctypes.byref(stats)))
            out.append((scene, handle, int(stats.bytes)))
        return out

    def pool_info(self) -> dict:
        info = _native.OlcPoolInfo()
        _native.check(self._lib, self._ctx, self._lib.olc_pool_info_get(self._ctx, ctypes.byref(info)))
        return {name: int(getattr(info, name)) for name, _ in info._fields_ if name != "reserved"}

    # -- batched and served rendering ---------------------------------------------
    def _job(self, request: RenderRequest, out, on_device: bool, sums=None) -> _native.OlcJob:
        width, height = int(request.width), int(request.height)
        if width <= 0 or height <= 0:
            raise ValueError("width and height must be positive")
        spp = self.config.samples_per_pixel if request.samples is None else int(request.samples)
        if not 1 <= spp <= 65536:
            raise ValueError("samples must be between 1 and 65536")
        bounces = 0 if request.max_bounces is None else int(request.max_bounces)
        if request.max_bounces is not None and not 1 <= bounces <= 64:
            raise ValueError("max_bounces must be between 1 and 64")
        frame_index = int(request.frame_index)
        if frame_index < 0:
            raise ValueError("frame_index cannot be negative")
        first_sample = int(request.first_sample)
        if first_sample < 0 or first_sample + spp > 0xFFFFFFFF:
            raise ValueError("first_sample must be non-negative and first_sample + samples below 2^32")
        job = _native.OlcJob()
        job.first_sample = first_sample
        job.scene = self.resident_scene(request.scene)
        job.width, job.height = width, height
        job.samples_per_pixel = spp
        job.frame_index = frame_index & 0xFFFFFFFF
        job.max_bounces = bounces
        job.camera = pack_camera(request.camera)
        job.out_rgba = _native.ptr(out).value
        job.out_sums = _native.ptr(sums).value
        job.out_is_device = 1 if on_device else 0
        return job

    def _record_timings(self, stats, total_ms, **extra):
        rays = stats.camera_rays + stats.extension_rays + stats.shadow_rays
        gpu_ms = float(stats.gpu_ms)
        self.last_timings = {
            "total_ms": total_ms,
            "gpu_ms": gpu_ms,
            "camera_rays": int(stats.camera_rays),
            "extension_rays": int(stats.extension_rays),
            "shadow_rays": int(stats.shadow_rays),
            "rays": int(rays),
            "closest_hit_rays": int(stats.camera_rays + stats.extension_rays),
            "mrays_per_s": rays / (gpu_ms * 1e3) if gpu_ms > 0 else 0.0,
            "queue_overflow": int(stats.overflow),
            "traversal_errors": int(stats.traversal_errors),
            "chunks": int(stats.chunks),
            "h2d_bytes": int(stats.h2d_bytes),
            "d2h_bytes": int(stats.d2h_bytes),
            **extra,
        }
        if stats.traversal_errors:
            raise RuntimeError(f"{stats.traversal_errors} traversal stack overflows")

    def render_batch(self, requests, outs=None, sums=None):
        """Render many requests as one wavefront (chunks of paths from several
        jobs and scenes share the ray queues; the chunk sequence replays from a
        CUDA graph when the same mix recurs).  Each image equals, bit for bit,
        ``render_frame`` of the same request on a fresh sequence.  Returns the
        list of (height, width, 4) float32 images (or fills ``outs``).
        ``sums`` (optional, one per request, same memory kind as the image):
        (height, width, 3) uint64/int64 buffers that receive the requests'
        fixed-point sample sums, which add exactly across shards of a frame
        (``ordinarylight_b200.distributed``)."""
        self._require_open()
        requests = list(requests)
        if outs is None:
            outs = [np.empty((int(r.height), int(r.width), 4), np.float32) for r in requests]
        if len(outs) != len(requests):
            raise ValueError("outs must match requests")
        t0 = time.perf_counter()
        if sums is not None and len(sums) != len(requests):
            raise ValueError("sums must match requests")
        jobs = (_native.OlcJob * max(len(requests), 1))()
        for k, (request, out) in enumerate(zip(requests, outs)):
            on_device = hasattr(out, "data_ptr") and getattr(out, "is_cuda", False)
            sm = None if sums is None else sums[k]
            if sm is not None:
                count = sm.numel() if hasattr(sm, "numel") else sm.size
                if count != int(request.width) * int(request.height) * 3:
                    raise ValueError("a sums buffer must hold height*width*3 64-bit values")
                if (hasattr(sm, "is_cuda") and sm.is_cuda) != on_device:
                    raise ValueError("sums and image buffers must both be on the device or both on the host")
            jobs[k] = self._job(request, out, on_device, sm)
        stats = _native.OlcRenderStats()
        _native.check(self._lib, self._ctx, self._lib.olc_render_batch(self._ctx, jobs, len(requests),
                                                                       ctypes.byref(stats)))
        self._record_timings(stats, (time.perf_counter() - t0) * 1e3, jobs=len(requests))
        return outs

    def submit(self, request: RenderRequest, out=None) -> int:
        """Queue a request for continuous batching; returns its ticket.  The
        request's paths join the shared wavefront at the next ``serve_step``."""
        self._require_open()
        if out is None:
            out = np.empty((int(request.height), int(request.width), 4), np.float32)
        on_device = hasattr(out, "data_ptr") and getattr(out, "is_cuda", False)
        job = self._job(request, out, on_device)
        ticket = ctypes.c_uint64()
        _native.check(self._lib, self._ctx, self._lib.olc_submit(self._ctx, ctypes.byref(job), ctypes.byref(ticket)))
        self._served_outputs[int(ticket.value)] = out
        return int(ticket.value)

    def serve_step(self):
        """Run one chunk of the queued requests; returns [(ticket, image)] of
        the requests it completed.  Statistics of the chunk land in
        ``last_timings``."""
        self._require_open()
        capacity = max(len(self._served_outputs), 1)
        done = (ctypes.c_uint64 * capacity)()
        count = ctypes.c_uint32()
        stats = _native.OlcRenderStats()
        t0 = time.perf_counter()
        status = self._lib.olc_serve_step(self._ctx, done, capacity, ctypes.byref(count), ctypes.byref(stats))
        if status != _native.OLC_OK:
            self._forget_dropped()
            _native.check(self._lib, self._ctx, status)
        self._record_timings(stats, (time.perf_counter() - t0) * 1e3, completed=int(count.value))
        return [(int(done[k]), self._served_outputs.pop(int(done[k]))) for k in range(count.value)]

    def queued_tickets(self):
        count = ctypes.c_uint32()
        _native.check(self._lib, self._ctx, self._lib.olc_queued_jobs(self._ctx, None, 0, ctypes.byref(count)))
        tickets = (ctypes.c_uint64 * max(count.value, 1))()
        _native.check(self._lib, self._ctx, self._lib.olc_queued_jobs(self._ctx, tickets, count.value,
                                                                      ctypes.byref(count)))
        return [int(tickets[k]) for k in range(count.value)]

    def _forget_dropped(self):
        queued = set(self.queued_tickets())
        for ticket in [t for t in self._served_outputs if t not in queued]:
            self._served_outputs.pop(ticket)

    def cancel(self, ticket: int) -> None:
        self._require_open()
        _native.check(self._lib, self._ctx, self._lib.olc_cancel(self._ctx, int(ticket)))
        self._served_outputs.pop(int(ticket), None)

    def job_bytes(self, request: RenderRequest) -> int:
        """Device bytes a queued request holds (its accumulator and output)."""
        job = _native.OlcJob()
        job.width, job.height = int(request.width), int(request.height)
        value = ctypes.c_uint64()
        _native.check(self._lib, self._ctx, self._lib.olc_job_bytes(self._ctx, ctypes.byref(job), ctypes.byref(value)))
        return int(value.value)

    # -- tracing primitives ---------------------------------------------------
    def trace_closest(self, scene, origins, directions, t_min=1e-4):
        """Closest hits of host rays: (instance_id uint32, primitive int32,
        t float32, barycentrics (n, 2) float32)."""
        import torch

        self._require_open()
        self._ensure_scene(scene)
        o = torch.as_tensor(np.ascontiguousarray(origins, np.float32).reshape(-1, 3), device=self.device)
        d = torch.as_tensor(np.ascontiguousarray(directions, np.float32).reshape(-1, 3), device=self.device)
        n = o.shape[0]
        inst = torch.empty(n, dtype=torch.int32, device=self.device)
        prim = torch.empty(n, dtype=torch.int32, device=self.device)
        t = torch.empty(n, dtype=torch.float32, device=self.device)
        bary = torch.empty((n, 2), dtype=torch.float32, device=self.device)
        torch.cuda.synchronize(self.device)
        _native.check(self._lib, self._ctx, self._lib.olc_trace_closest(
            self._ctx, n, _native.ptr(o), _native.ptr(d), float(t_min), _native.ptr(inst), _native.ptr(prim),
            _native.ptr(t), _native.ptr(bary)))
        return (inst.cpu().numpy().view(np.uint32), prim.cpu().numpy(), t.cpu().numpy(), bary.cpu().numpy())

    def trace_occluded(self, scene, origins, directions, t_max, t_min=1e-3):
        import torch

        self._require_open()
        self._ensure_scene(scene)
        o = torch.as_tensor(np.ascontiguousarray(origins, np.float32).reshape(-1, 3), device=self.device)
        d = torch.as_tensor(np.ascontiguousarray(directions, np.float32).reshape(-1, 3), device=self.device)
        tm = torch.as_tensor(np.ascontiguousarray(t_max, np.float32).reshape(-1), device=self.device)
        occ = torch.empty(o.shape[0], dtype=torch.uint8, device=self.device)
        torch.cuda.synchronize(self.device)
        _native.check(self._lib, self._ctx, self._lib.olc_trace_occluded(
            self._ctx, o.shape[0], _native.ptr(o), _native.ptr(d), float(t_min), _native.ptr(tm), _native.ptr(occ)))
        return occ.cpu().numpy().astype(bool)

    def camera_rays(self, camera, width, height, *, sample=0, frame_index=0, jitter=None):
        """Device camera rays of one sample (the model of the camera rays that bounce-0 traversal generates)."""
        import torch

        self._require_open()
        n = int(width) * int(height)
        o = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        d = torch.empty((n, 3), dtype=torch.float32, device=self.device)
        j = None if jitter is None else np.ascontiguousarray(jitter, np.float32)
        cam = pack_camera(camera)
        _native.check(self._lib, self._ctx, self._lib.olc_camera_rays(
            self._ctx, ctypes.byref(cam), int(width), int(height), int(sample), int(frame_index),
            _native.ptr(j), _native.ptr(o), _native.ptr(d)))
        return o.cpu().numpy(), d.cpu().numpy()

    def bvh_info(self):
        info = _native.OlcBvhInfo()
        _native.check(self._lib, self._ctx, self._lib.olc_bvh_info_get(self._ctx, ctypes.byref(info)))
        return {"blas_count": info.blas_count, "blas_nodes": info.blas_nodes, "tlas_nodes": info.tlas_nodes,
                "triangles": info.triangles, "build_ms": info.build_ms}

    def validate_bvh(self, scene) -> int:
        self._require_open()
        self._ensure_scene(scene)
        bad = ctypes.c_uint64()
        _native.check(self._lib, self._ctx, self._lib.olc_bvh_validate(self._ctx, ctypes.byref(bad)))
        return int(bad.value)

    # -- sequencing / configuration ----------------------------------------------
    def reset_output_history(self):
        """Forget temporal (ReSTIR) history; called by Renderer.reset_sequence
        (ordinarylight/renderer/_core.py:339-351)."""
        self._require_open()
        self._output_history = None
        _native.check(self._lib, self._ctx, self._lib.olc_reset_history(self._ctx))

    reset_accumulation = reset_output_history

    def reconfigure(self, **changes):
        """Apply configuration changes in place (Renderer.reconfigure,
        ordinarylight/renderer/_core.py:386-413)."""
        self._require_open()
        names = {f.name for f in fields(CudaRendererConfig)}
        unknown = set(changes) - names
        if unknown:
            raise RuntimeError(f"unsupported settings {sorted(unknown)} require renderer recreation")
        if "device" in changes and int(changes["device"]) != self.config.device:
            raise RuntimeError("changing the device requires renderer recreation")
        config = replace(self.config, **changes)
        _native.check(self._lib, self._ctx, self._lib.olc_reconfigure(self._ctx, ctypes.byref(config.native())))
        self.config = config
        return config

    def close(self):
        if self._closed:
            return
        self._closed = True
        ctx, self._ctx = self._ctx, None
        if ctx:
            self._lib.olc_destroy(ctx)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        self._require_open()
        return self

    def __exit__(self, *_exc):
        self.close()


def config_dict(config: CudaRendererConfig) -> dict:
    return asdict(config)


__all__ = ["CudaRendererConfig", "CudaWavefrontRenderer", "RenderRequest"]
