"""Denoiser input signals of the wavefront path (the canonical contract of
ordinarylight/denoising/signals.py:25-140), for environments without the
reference package.  When the reference is importable,
``CudaWavefrontRenderer.capture_denoiser_signals`` returns its own
``DenoiserSignals`` instead; these classes mirror their fields and checks.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


class SignalValidationError(ValueError):
    """A denoiser input violates the canonical contract."""


def _matrix(value, name):
    result = np.ascontiguousarray(value, dtype=np.float32)
    if result.shape != (4, 4) or not np.isfinite(result).all():
        raise SignalValidationError(f"{name} must be a finite 4x4 matrix")
    return result


@dataclass(frozen=True)
class DenoiserFrameInfo:
    """World-to-clip matrices of this and the previous frame, the frame
    index, sub-pixel jitters and whether temporal history is cut."""

    world_to_clip: np.ndarray
    previous_world_to_clip: np.ndarray
    frame_index: int
    jitter: tuple = (0.0, 0.0)
    previous_jitter: tuple = (0.0, 0.0)
    camera_cut: bool = False

    def __post_init__(self):
        object.__setattr__(self, "world_to_clip", _matrix(self.world_to_clip, "world_to_clip"))
        object.__setattr__(self, "previous_world_to_clip",
                           _matrix(self.previous_world_to_clip, "previous_world_to_clip"))
        if int(self.frame_index) < 0:
            raise SignalValidationError("frame_index cannot be negative")
        object.__setattr__(self, "frame_index", int(self.frame_index))


@dataclass(frozen=True)
class DenoiserSignals:
    """Diffuse and specular radiance with hit distance (w), world normal and
    roughness, linear view depth, motion to the previous frame in pixels
    (+x right, +y down) and material ids, with the frame's camera info."""

    diffuse_radiance_hit_distance: np.ndarray
    specular_radiance_hit_distance: np.ndarray
    normal_roughness: np.ndarray
    view_z: np.ndarray
    motion: np.ndarray
    material_id: np.ndarray
    frame: DenoiserFrameInfo

    def __post_init__(self):
        view_z = np.asarray(self.view_z)
        if view_z.ndim != 2 or min(view_z.shape) < 1:
            raise SignalValidationError("view_z must have shape (height, width)")
        h, w = view_z.shape
        shapes = {"diffuse_radiance_hit_distance": (h, w, 4), "specular_radiance_hit_distance": (h, w, 4),
                  "normal_roughness": (h, w, 4), "view_z": (h, w), "motion": (h, w, 2), "material_id": (h, w)}
        for name, shape in shapes.items():
            value = np.asarray(getattr(self, name))
            dtype = np.uint32 if name == "material_id" else np.float32
            if value.dtype != dtype or value.shape != shape:
                raise SignalValidationError(f"{name} must be {np.dtype(dtype)} of shape {shape}")
            if value.dtype == np.float32 and not np.isfinite(value).all():
                raise SignalValidationError(f"{name} must contain finite values")
            object.__setattr__(self, name, np.ascontiguousarray(value))
        if np.any(self.diffuse_radiance_hit_distance[..., 3] < 0.0) or \
                np.any(self.specular_radiance_hit_distance[..., 3] < 0.0):
            raise SignalValidationError("hit distances cannot be negative")
        rough = self.normal_roughness[..., 3]
        if np.any((rough < 0.0) | (rough > 1.0)):
            raise SignalValidationError("roughness must be in [0, 1]")

    @property
    def extent(self):
        return self.view_z.shape[1], self.view_z.shape[0]


def camera_matrix(camera, width: int, height: int) -> np.ndarray:
    """OpenGL-style world-to-clip matrix of a perspective or orthographic
    camera (near 0.01, far 10000), the convention of the reference's
    raster camera_matrix (ordinarylight/raster/_core.py:979-999)."""
    eye = np.asarray(camera.position, np.float32)
    forward = np.asarray(camera.target, np.float32) - eye
    forward /= np.linalg.norm(forward)
    right = np.cross(forward, np.asarray(camera.up, np.float32))
    right /= np.linalg.norm(right)
    up = np.cross(right, forward)
    view = np.eye(4, dtype=np.float32)
    view[:3, :3] = np.stack((right, up, -forward))
    view[:3, 3] = -view[:3, :3] @ eye
    aspect, near, far = width / height, 0.01, 10000.0
    if hasattr(camera, "vertical_size"):
        top = camera.vertical_size * 0.5
        proj = np.diag([1.0 / (top * aspect), 1.0 / top, -2.0 / (far - near), 1.0]).astype(np.float32)
        proj[2, 3] = -(far + near) / (far - near)
    elif hasattr(camera, "vertical_fov_degrees"):
        f = 1.0 / np.tan(np.radians(camera.vertical_fov_degrees) * 0.5)
        proj = np.zeros((4, 4), np.float32)
        proj[0, 0], proj[1, 1] = f / aspect, f
        proj[2, 2], proj[2, 3] = -(far + near) / (far - near), -2.0 * far * near / (far - near)
        proj[3, 2] = -1.0
    else:
        raise ValueError("panoramic cameras require a non-linear raster projection")
    return proj @ view


__all__ = ["DenoiserFrameInfo", "DenoiserSignals", "SignalValidationError", "camera_matrix"]
