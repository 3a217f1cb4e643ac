"""ctypes binding of libolcuda.so (declarations in include/olcuda.h).

The library is built in-tree (``ordinarylight_b200/_lib/libolcuda.so``) by
``ordinarylight_b200.build``.  Loading fails loudly when it is missing: the
renderer has no CPU fallback.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_float, c_int, c_int32, c_uint8, c_uint32, c_uint64, c_void_p, c_double
from pathlib import Path
import threading

LIBRARY_PATH = Path(__file__).resolve().parent / "_lib" / "libolcuda.so"

OLC_OK = 0
OLC_ERR_VALUE = 1
OLC_ERR_TYPE = 2
OLC_ERR_RUNTIME = 3
OLC_ERR_CUDA = 4
OLC_ERR_MEMORY = 5
OLC_ERR_CLOSED = 6
OLC_ERR_TIMEOUT = 7

MODE_PRODUCTION = 0
MODE_REFERENCE_COMPATIBLE = 1
PROJECTION_PERSPECTIVE = 0
PROJECTION_ORTHOGRAPHIC = 1
PROJECTION_PANORAMIC = 2
ENV_NONE = 0
ENV_CONSTANT = 1
ENV_EQUIRECT = 2
DEFAULT_SCENE = 0xFFFFFFFF

_f32p = POINTER(c_float)
_u32p = POINTER(c_uint32)


class OlcConfig(ctypes.Structure):
    _fields_ = [
        ("device", c_int32), ("mode", c_uint32), ("max_bounces", c_uint32), ("seed", c_uint32),
        ("russian_roulette_start", c_uint32), ("russian_roulette_min_survival", c_float),
        ("restir", c_uint32), ("restir_candidates", c_uint32), ("restir_temporal", c_uint32),
        ("restir_spatial", c_uint32), ("restir_neighbours", c_uint32), ("restir_radius", c_float),
        ("restir_max_history", c_uint32), ("block_size", c_uint32), ("stack_depth", c_uint32),
        ("chunk_paths", c_uint32), ("use_graphs", c_uint32), ("flatten_instances", c_uint32),
        ("trace_scheduler", c_uint32), ("disable_nee", c_uint32), ("trace_block", c_uint32),
        ("ray_sort", c_uint32), ("serve_aging_steps", c_uint32), ("sample_variance", c_uint32),
        ("reserved", c_uint32 * 1),
    ]


class OlcSceneDesc(ctypes.Structure):
    _fields_ = [
        ("num_meshes", c_uint32), ("mesh_vertex_offset", _u32p), ("mesh_triangle_offset", _u32p),
        ("vertices", _f32p), ("normals", _f32p), ("indices", _u32p),
        ("num_instances", c_uint32), ("instance_object_to_world", _f32p), ("instance_mesh", _u32p),
        ("instance_material", _u32p), ("instance_id", _u32p), ("instance_primitive_offset", _u32p),
        ("num_materials", c_uint32), ("materials", _f32p),
        ("num_emitters", c_uint32), ("emitters", _f32p), ("emissive_weight", c_float),
        ("num_lights", c_uint32), ("lights", _f32p),
        ("environment_kind", c_uint32), ("environment_color", c_float * 3), ("environment_rotation", c_float),
        ("environment_width", c_uint32), ("environment_height", c_uint32), ("environment_image", _f32p),
        ("volume_present", c_uint32), ("volume_dims", c_uint32 * 3), ("volume_density", _f32p),
        ("volume_world_to_box", c_float * 12), ("volume_sigma_t_scale", c_float), ("volume_albedo", c_float),
        ("volume_max_density", c_float), ("reserved", c_uint32 * 7),
        ("texcoords", _f32p), ("tangents", _f32p), ("num_texture_words", c_uint32), ("texture_words", _u32p),
        ("num_texture_bindings", c_uint32), ("texture_bindings", _f32p), ("material_textures", _f32p),
        ("num_ref_volumes", c_uint32), ("ref_volume_records", _f32p), ("ref_grid_values", c_uint64),
        ("ref_volume_grids", _f32p), ("ref_lut_entries", c_uint64), ("ref_volume_luts", _f32p),
    ]


class OlcCamera(ctypes.Structure):
    _fields_ = [
        ("position", c_float * 3), ("forward", c_float * 3), ("right", c_float * 3), ("up", c_float * 3),
        ("half_height", c_float), ("horizontal_half", c_float), ("vertical_half", c_float),
        ("projection", c_uint32),
    ]


class OlcRenderStats(ctypes.Structure):
    _fields_ = [
        ("camera_rays", c_uint64), ("extension_rays", c_uint64), ("shadow_rays", c_uint64),
        ("overflow", c_uint64), ("traversal_errors", c_uint64), ("gpu_ms", c_float),
        ("raygen_ms", c_float), ("trace_ms", c_float), ("shade_ms", c_float), ("shadow_ms", c_float),
        ("restir_ms", c_float), ("accumulate_ms", c_float), ("chunks", c_uint32),
        ("restir_history_used", c_uint32), ("jobs_completed", c_uint32), ("reserved", c_uint32),
        ("h2d_bytes", c_uint64), ("d2h_bytes", c_uint64),
    ]


class OlcBvhInfo(ctypes.Structure):
    _fields_ = [
        ("blas_count", c_uint32), ("blas_nodes", c_uint32), ("tlas_nodes", c_uint32), ("triangles", c_uint32),
        ("max_depth", c_uint32), ("reserved", c_uint32 * 3), ("build_ms", c_double),
    ]


class OlcLaunchRecord(ctypes.Structure):
    _fields_ = [
        ("stage", c_uint32), ("bounce", c_uint32), ("chunk", c_uint32), ("misses", c_uint32),
        ("items", c_uint64), ("ms", c_float), ("reserved", c_uint32),
    ]


class OlcSceneStats(ctypes.Structure):
    _fields_ = [
        ("bytes", c_uint64), ("triangles", c_uint32), ("blas_count", c_uint32), ("blas_nodes", c_uint32),
        ("tlas_nodes", c_uint32), ("flattened_instances", c_uint32), ("reserved", c_uint32), ("build_ms", c_double),
    ]


class OlcPoolInfo(ctypes.Structure):
    _fields_ = [
        ("resident_scenes", c_uint32), ("queued_jobs", c_uint32), ("scene_bytes", c_uint64),
        ("pool_bytes", c_uint64), ("wavefront_bytes", c_uint64), ("pixel_bytes", c_uint64),
        ("pixel_bytes_used", c_uint64), ("reserved", c_uint64 * 3),
    ]


class OlcMotionCamera(ctypes.Structure):
    _fields_ = [("origin", c_double * 3), ("forward", c_double * 3), ("right", c_double * 3), ("up", c_double * 3),
                ("scale", c_double)]


class OlcMotionMesh(ctypes.Structure):
    _fields_ = [("first", c_uint32), ("count", c_uint32), ("previous_first", c_uint32), ("reserved", c_uint32)]


class OlcJob(ctypes.Structure):
    _fields_ = [
        ("scene", c_uint32), ("width", c_uint32), ("height", c_uint32), ("samples_per_pixel", c_uint32),
        ("frame_index", c_uint32), ("max_bounces", c_uint32), ("first_sample", c_uint32), ("reserved", c_uint32),
        ("camera", OlcCamera), ("out_rgba", c_void_p), ("out_sums", c_void_p), ("out_is_device", c_int32),
        ("reserved2", c_uint32),
    ]


STAGE_NAMES = ("raygen", "trace_closest", "restir", "shade", "trace_shadow", "accumulate", "resolve", "sort")


# Exported symbols and their signatures (argument types, all return int
# unless listed otherwise).
_SIGNATURES = {
    "olc_abi_version": ([], c_int),
    "olc_last_error": ([c_void_p], c_char_p),
    "olc_create": ([POINTER(OlcConfig), POINTER(c_void_p)], c_int),
    "olc_destroy": ([c_void_p], c_int),
    "olc_reconfigure": ([c_void_p, POINTER(OlcConfig)], c_int),
    "olc_upload_scene": ([c_void_p, POINTER(OlcSceneDesc)], c_int),
    "olc_scene_bytes": ([c_void_p, POINTER(c_uint64)], c_int),
    "olc_add_scene": ([c_void_p, POINTER(OlcSceneDesc), POINTER(c_uint32)], c_int),
    "olc_remove_scene": ([c_void_p, c_uint32], c_int),
    "olc_update_scene": ([c_void_p, c_uint32, POINTER(OlcSceneDesc), c_void_p, POINTER(c_int32), POINTER(c_uint32)],
                         c_int),
    "olc_scene_stats_get": ([c_void_p, c_uint32, POINTER(OlcSceneStats)], c_int),
    "olc_pool_info_get": ([c_void_p, POINTER(OlcPoolInfo)], c_int),
    "olc_render_batch": ([c_void_p, POINTER(OlcJob), c_uint32, POINTER(OlcRenderStats)], c_int),
    "olc_submit": ([c_void_p, POINTER(OlcJob), POINTER(c_uint64)], c_int),
    "olc_serve_step": ([c_void_p, POINTER(c_uint64), c_uint32, POINTER(c_uint32), POINTER(OlcRenderStats)], c_int),
    "olc_cancel": ([c_void_p, c_uint64], c_int),
    "olc_queued_jobs": ([c_void_p, POINTER(c_uint64), c_uint32, POINTER(c_uint32)], c_int),
    "olc_job_bytes": ([c_void_p, POINTER(OlcJob), POINTER(c_uint64)], c_int),
    "olc_render": ([c_void_p, POINTER(OlcCamera), c_uint32, c_uint32, c_uint32, c_uint32, c_void_p, c_int,
                    POINTER(OlcRenderStats)], c_int),
    "olc_read_products": ([c_void_p, c_uint32, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "olc_read_variance": ([c_void_p, c_uint32, c_uint32, c_void_p, c_int], c_int),
    "olc_read_hit_geometry": ([c_void_p, c_uint32, c_uint32, c_void_p, c_void_p], c_int),
    "olc_capture_motion_state": ([c_void_p], c_int),
    "olc_read_path_signals": ([c_void_p, c_uint32, c_uint32, c_void_p, c_void_p], c_int),
    "olc_sample_texture": ([c_void_p, c_uint32, c_int32, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                            c_void_p], c_int),
    "olc_read_motion": ([c_void_p, c_uint32, c_uint32, POINTER(OlcMotionMesh), c_uint32, POINTER(OlcMotionCamera),
                         POINTER(OlcMotionCamera), c_void_p], c_int),
    "olc_reset_history": ([c_void_p], c_int),
    "olc_trace_closest": ([c_void_p, c_uint32, c_void_p, c_void_p, c_float, c_void_p, c_void_p, c_void_p,
                           c_void_p], c_int),
    "olc_trace_occluded": ([c_void_p, c_uint32, c_void_p, c_void_p, c_float, c_void_p, c_void_p], c_int),
    "olc_camera_rays": ([c_void_p, POINTER(OlcCamera), c_uint32, c_uint32, c_uint32, c_uint32, c_void_p,
                         c_void_p, c_void_p], c_int),
    "olc_morton_codes": ([c_void_p, c_uint32, c_void_p, c_void_p], c_int),
    "olc_radix_sort_pairs": ([c_void_p, c_uint32, c_uint32, c_void_p, c_void_p], c_int),
    "olc_radix_sort_pairs_noalloc": ([c_uint32, c_uint32, c_void_p, c_void_p, c_void_p], c_int),
    "olc_bvh_info_get": ([c_void_p, POINTER(OlcBvhInfo)], c_int),
    "olc_bvh_validate": ([c_void_p, POINTER(c_uint64)], c_int),
    "olc_frame_profile": ([c_void_p, POINTER(OlcLaunchRecord), c_uint32, POINTER(c_uint32)], c_int),
    "olc_stream": ([c_void_p, POINTER(c_void_p)], c_int),
}

EXPORTED_SYMBOLS = tuple(_SIGNATURES)

_lock = threading.Lock()
_lib = None


class NativeLibraryMissing(RuntimeError):
    """libolcuda.so is not built (run ordinarylight_b200.build.build())."""


def load(path: Path | None = None):
    """Load libolcuda.so once and declare every entry point."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        target = Path(path) if path is not None else LIBRARY_PATH
        if not target.exists():
            raise NativeLibraryMissing(
                f"{target} is missing; build it with `python -m ordinarylight_b200.build` "
                "(the CUDA renderer has no CPU fallback)")
        lib = ctypes.CDLL(str(target))
        for name, (argtypes, restype) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = restype
        if path is None:
            _lib = lib
        return lib


def error_message(lib, ctx) -> str:
    raw = lib.olc_last_error(ctx)
    return raw.decode("utf-8", "replace") if raw else "unknown error"


def check(lib, ctx, status: int):
    """Map an olc_status to the exception types the reference raises."""
    if status == OLC_OK:
        return
    message = error_message(lib, ctx)
    if status == OLC_ERR_VALUE:
        raise ValueError(message)
    if status == OLC_ERR_TYPE:
        raise TypeError(message)
    if status == OLC_ERR_MEMORY:
        raise MemoryError(message)
    if status == OLC_ERR_TIMEOUT:
        raise TimeoutError(message)
    raise RuntimeError(message)


def ptr(array) -> c_void_p:
    """Address of a contiguous numpy array, a torch tensor, or None."""
    if array is None:
        return c_void_p(0)
    if hasattr(array, "data_ptr"):
        return c_void_p(array.data_ptr())
    return c_void_p(array.ctypes.data)


def typed_ptr(array, ctype):
    if array is None:
        return ctypes.cast(c_void_p(0), POINTER(ctype))
    return array.ctypes.data_as(POINTER(ctype))
