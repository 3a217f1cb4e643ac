"""Host scene model: the subset of OrdinaryLight's backend-neutral scene API
that the wavefront path consumes.

The CUDA renderer reads scenes structurally (``visible_meshes``, each mesh's
``vertices``/``indices``/``normals``/``transform``/``material``/``resource``/
``id``, ``lights``, ``environment``, ``visible_volumes``, ``revision``), so it
accepts the reference's own ``ordinarylight.Scene`` unchanged.  This module
supplies the same names and semantics for environments without the reference
package installed:

* ``Transform``   ordinarylight/scene/_core.py:50-114
* ``Material``    ordinarylight/scene/_core.py:431-553 (parameters the
                  wavefront path shades with; the rest are accepted and kept)
* ``Mesh`` / ``MeshResource`` / ``Instance``  :556-815
* ``Scene``       :943-3093 (mesh/instance/light/environment/volume
                  membership, stable ids, revision counters, packing helpers)
* cameras         ordinarylight/cameras/*.py
* lights          ordinarylight/lights/*.py
"""

from __future__ import annotations

from dataclasses import dataclass, field
import math
from types import MappingProxyType

import numpy as np

__all__ = [
    "Transform", "Material", "Texture", "TextureTransform", "Mesh", "MeshResource", "Instance", "Scene",
    "Volume", "VolumeMaterial", "Texture1D",
    "PerspectiveCamera", "OrthographicCamera", "PanoramicCamera",
    "PointLight", "DirectionalLight", "SpotLight", "EnvironmentLight",
    "CAMERA_TYPES", "LIGHT_TYPES",
]

_LUMINANCE = (0.2126, 0.7152, 0.0722)


def _vec3(value, name):
    result = np.asarray(value, dtype=np.float32)
    if result.shape != (3,):
        raise ValueError(f"{name} must contain exactly three values")
    if not np.all(np.isfinite(result)):
        raise ValueError(f"{name} must be finite")
    return result


# ---------------------------------------------------------------------------
# cameras (ordinarylight/cameras/)
# ---------------------------------------------------------------------------
def _validate_look_at(position, target, up):
    p, t, u = _vec3(position, "position"), _vec3(target, "target"), _vec3(up, "up")
    forward = t - p
    if float(np.linalg.norm(forward)) < 1e-8:
        raise ValueError("camera position and target must differ")
    if float(np.linalg.norm(np.cross(forward, u))) < 1e-8:
        raise ValueError("camera up vector must not be parallel to the view direction")


@dataclass(frozen=True)
class PerspectiveCamera:
    """Pinhole camera (ordinarylight/cameras/perspective_camera.py:8-20)."""

    position: tuple
    target: tuple
    up: tuple = (0.0, 1.0, 0.0)
    vertical_fov_degrees: float = 45.0

    def __post_init__(self):
        _validate_look_at(self.position, self.target, self.up)
        if not 1.0 <= self.vertical_fov_degrees < 179.0:
            raise ValueError("vertical_fov_degrees must be in [1, 179)")


@dataclass(frozen=True)
class OrthographicCamera:
    """Parallel projection (ordinarylight/cameras/orthographic_camera.py)."""

    position: tuple
    target: tuple
    up: tuple = (0.0, 1.0, 0.0)
    vertical_size: float = 2.0

    def __post_init__(self):
        _validate_look_at(self.position, self.target, self.up)
        if not np.isfinite(self.vertical_size) or self.vertical_size <= 0.0:
            raise ValueError("vertical_size must be finite and positive")

    @property
    def vertical_fov_degrees(self):
        return 90.0


@dataclass(frozen=True)
class PanoramicCamera:
    """Equirectangular camera (ordinarylight/cameras/panoramic_camera.py)."""

    position: tuple
    target: tuple
    up: tuple = (0.0, 1.0, 0.0)
    horizontal_fov_degrees: float = 360.0
    vertical_fov_degrees: float = 180.0

    def __post_init__(self):
        _validate_look_at(self.position, self.target, self.up)
        if not 1.0 <= self.horizontal_fov_degrees <= 360.0:
            raise ValueError("horizontal_fov_degrees must be in [1, 360]")
        if not 1.0 <= self.vertical_fov_degrees <= 180.0:
            raise ValueError("vertical_fov_degrees must be in [1, 180]")


CAMERA_TYPES = (PerspectiveCamera, OrthographicCamera, PanoramicCamera)


# ---------------------------------------------------------------------------
# lights (ordinarylight/lights/)
# ---------------------------------------------------------------------------
def _validate_color_intensity(color, intensity):
    c = _vec3(color, "color")
    if np.any(c < 0.0):
        raise ValueError("color components cannot be negative")
    if not math.isfinite(intensity) or intensity < 0.0:
        raise ValueError("intensity must be finite and non-negative")


@dataclass
class PointLight:
    position: tuple
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 1.0
    range: float | None = None
    id: int | None = field(default=None, init=False)

    def __post_init__(self):
        _vec3(self.position, "position")
        _validate_color_intensity(self.color, self.intensity)
        if self.range is not None and not (self.range > 0.0):
            raise ValueError("range must be positive")


@dataclass
class DirectionalLight:
    direction: tuple
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 1.0
    id: int | None = field(default=None, init=False)

    def __post_init__(self):
        if float(np.linalg.norm(_vec3(self.direction, "direction"))) < 1e-8:
            raise ValueError("direction cannot be zero")
        _validate_color_intensity(self.color, self.intensity)


@dataclass
class SpotLight:
    position: tuple
    direction: tuple
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 1.0
    inner_cone_angle: float = 0.0
    outer_cone_angle: float = math.pi / 4.0
    range: float | None = None
    id: int | None = field(default=None, init=False)

    def __post_init__(self):
        _vec3(self.position, "position")
        if float(np.linalg.norm(_vec3(self.direction, "direction"))) < 1e-8:
            raise ValueError("direction cannot be zero")
        _validate_color_intensity(self.color, self.intensity)
        if not 0.0 <= self.inner_cone_angle <= self.outer_cone_angle:
            raise ValueError("inner_cone_angle must be in [0, outer_cone_angle]")
        if not 0.0 < self.outer_cone_angle <= math.pi / 2.0:
            raise ValueError("outer_cone_angle must be in (0, pi/2]")


@dataclass(frozen=True)
class EnvironmentLight:
    """Constant or equirectangular environment (lights/environment_light.py)."""

    image: np.ndarray | None = field(default=None, compare=False, repr=False)
    color: tuple = (1.0, 1.0, 1.0)
    intensity: float = 1.0
    rotation: float = 0.0

    def __post_init__(self):
        _validate_color_intensity(self.color, self.intensity)
        if not math.isfinite(self.rotation):
            raise ValueError("environment rotation must be finite")
        if self.image is None:
            return
        image = np.array(self.image, dtype=np.float32, copy=True, order="C")
        if image.ndim != 3 or image.shape[2] not in (3, 4) or min(image.shape[:2]) < 1:
            raise ValueError("environment image must have shape (height, width, 3 or 4)")
        image = np.ascontiguousarray(image[..., :3])
        if not np.all(np.isfinite(image)) or np.any(image < 0.0):
            raise ValueError("environment image radiance must be finite and non-negative")
        image.flags.writeable = False
        object.__setattr__(self, "image", image)


LIGHT_TYPES = (PointLight, DirectionalLight, SpotLight)


# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class Transform:
    """Immutable affine object-to-world transform (scene/_core.py:50-114)."""

    matrix: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32), compare=False, repr=False)

    def __post_init__(self):
        m = np.array(self.matrix, dtype=np.float32, copy=True)
        if m.shape != (4, 4):
            raise ValueError("transform matrix must have shape (4, 4)")
        if not np.all(np.isfinite(m)):
            raise ValueError("transform matrix must contain finite values")
        if not np.allclose(m[3], (0.0, 0.0, 0.0, 1.0), atol=1e-6):
            raise ValueError("transform matrix must be affine")
        if abs(float(np.linalg.det(m[:3, :3]))) < 1e-10:
            raise ValueError("transform linear component must be invertible")
        m.setflags(write=False)
        object.__setattr__(self, "matrix", m)

    @classmethod
    def translation(cls, offset):
        m = np.eye(4, dtype=np.float32)
        m[:3, 3] = _vec3(offset, "translation")
        return cls(m)

    @classmethod
    def scale(cls, factors):
        v = np.asarray(factors, dtype=np.float32)
        if v.ndim == 0:
            v = np.repeat(v, 3)
        m = np.eye(4, dtype=np.float32)
        m[:3, :3] = np.diag(_vec3(v, "scale"))
        return cls(m)

    @classmethod
    def rotation(cls, axis, angle_radians):
        """Rotation about ``axis`` (Rodrigues' formula)."""
        a = _vec3(axis, "rotation axis").astype(np.float64)
        n = float(np.linalg.norm(a))
        if n < 1e-8:
            raise ValueError("rotation axis cannot be zero")
        a /= n
        k = np.array([[0.0, -a[2], a[1]], [a[2], 0.0, -a[0]], [-a[1], a[0], 0.0]])
        r = np.eye(3) + math.sin(angle_radians) * k + (1.0 - math.cos(angle_radians)) * (k @ k)
        m = np.eye(4, dtype=np.float32)
        m[:3, :3] = r
        return cls(m)

    def __matmul__(self, other):
        if not isinstance(other, Transform):
            return NotImplemented
        return Transform(self.matrix @ other.matrix)


@dataclass(frozen=True)
class Texture:
    """Decoded RGBA8 texture with glTF sampler state (scene/_core.py:115-135)."""

    pixels: np.ndarray = field(compare=False, repr=False)
    wrap_s: str = "repeat"
    wrap_t: str = "repeat"
    linear_filter: bool = True

    def __post_init__(self):
        pixels = np.ascontiguousarray(self.pixels, dtype=np.uint8)
        if pixels.ndim != 3 or pixels.shape[2] != 4 or min(pixels.shape[:2]) < 1:
            raise ValueError("texture pixels must have shape (height, width, 4)")
        for name in ("wrap_s", "wrap_t"):
            if getattr(self, name) not in {"repeat", "clamp", "mirror"}:
                raise ValueError(f"{name} must be repeat, clamp, or mirror")
        pixels.flags.writeable = False
        object.__setattr__(self, "pixels", pixels)


@dataclass(frozen=True)
class TextureTransform:
    """KHR_texture_transform UV mapping (scene/_core.py:402-428)."""

    offset: tuple = (0.0, 0.0)
    scale: tuple = (1.0, 1.0)
    rotation: float = 0.0
    texcoord_set: int = 0

    def __post_init__(self):
        offset = tuple(float(v) for v in self.offset)
        scale = tuple(float(v) for v in self.scale)
        if len(offset) != 2 or len(scale) != 2:
            raise ValueError("texture transform offset and scale must be vec2 values")
        if not np.all(np.isfinite((*offset, *scale, float(self.rotation)))):
            raise ValueError("texture transform values must be finite")
        if abs(scale[0]) < 1e-8 or abs(scale[1]) < 1e-8:
            raise ValueError("texture transform scale components cannot be zero")
        if int(self.texcoord_set) not in (0, 1):
            raise ValueError("texcoord_set must be zero or one")
        object.__setattr__(self, "offset", offset)
        object.__setattr__(self, "scale", scale)
        object.__setattr__(self, "rotation", float(self.rotation))
        object.__setattr__(self, "texcoord_set", int(self.texcoord_set))


_TEXTURE_SLOTS = ("base_color", "metallic_roughness", "emissive", "normal", "occlusion", "transmission")


@dataclass(frozen=True)
class Material:
    """PBR material (scene/_core.py:431-553): the parameters and textures the
    wavefront shades (base colour, metallic-roughness, emissive, normal,
    occlusion and transmission maps, each with a KHR texture transform)."""

    base_color: tuple = (0.8, 0.8, 0.8)
    emission: tuple = (0.0, 0.0, 0.0)
    metallic: float = 0.0
    roughness: float = 1.0
    transmission: float = 0.0
    ior: float = 1.5
    opacity: float = 1.0
    emission_two_sided: bool = False
    base_color_texture: Texture | None = field(default=None, compare=False)
    metallic_roughness_texture: Texture | None = field(default=None, compare=False)
    emissive_texture: Texture | None = field(default=None, compare=False)
    normal_texture: Texture | None = field(default=None, compare=False)
    normal_scale: float = 1.0
    occlusion_texture: Texture | None = field(default=None, compare=False)
    occlusion_strength: float = 1.0
    transmission_texture: Texture | None = field(default=None, compare=False)
    base_color_transform: TextureTransform = field(default_factory=TextureTransform)
    metallic_roughness_transform: TextureTransform = field(default_factory=TextureTransform)
    emissive_transform: TextureTransform = field(default_factory=TextureTransform)
    normal_transform: TextureTransform = field(default_factory=TextureTransform)
    occlusion_transform: TextureTransform = field(default_factory=TextureTransform)
    transmission_transform: TextureTransform = field(default_factory=TextureTransform)

    def __post_init__(self):
        for slot in _TEXTURE_SLOTS:
            texture = getattr(self, f"{slot}_texture")
            if texture is not None and not isinstance(texture, Texture):
                raise TypeError(f"{slot}_texture must be a Texture")
            if not isinstance(getattr(self, f"{slot}_transform"), TextureTransform):
                raise TypeError(f"{slot}_transform must be a TextureTransform")
        if self.normal_scale < 0.0:
            raise ValueError("normal_scale cannot be negative")
        if not 0.0 <= self.occlusion_strength <= 1.0:
            raise ValueError("occlusion_strength must be between zero and one")
        color = _vec3(self.base_color, "base_color")
        emission = _vec3(self.emission, "emission")
        if np.any(color < 0.0) or np.any(color > 1.0):
            raise ValueError("base_color components must be between zero and one")
        if np.any(emission < 0.0):
            raise ValueError("emission components cannot be negative")
        for name in ("metallic", "roughness", "transmission", "opacity"):
            if not 0.0 <= getattr(self, name) <= 1.0:
                raise ValueError(f"{name} must be between zero and one")
        if self.ior <= 0.0:
            raise ValueError("ior must be positive")
        if not isinstance(self.emission_two_sided, bool):
            raise TypeError("emission_two_sided must be a bool")


def _generate_tangents(vertices, indices, normals, texcoords):
    """Per-vertex tangents from UV gradients, orthogonalised against the
    normal, with handedness from the accumulated bitangent; an axis-derived
    tangent where the UVs are degenerate (Mesh._generate_tangents,
    scene/_core.py:740-772)."""
    vertices = np.asarray(vertices, np.float32)
    tri = vertices[indices]
    uv = np.asarray(texcoords, np.float32)[indices]
    edge_a, edge_b = tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]
    uv_a, uv_b = uv[:, 1] - uv[:, 0], uv[:, 2] - uv[:, 0]
    det = uv_a[:, 0] * uv_b[:, 1] - uv_a[:, 1] * uv_b[:, 0]
    ok = np.abs(det) >= 1e-10
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0).astype(np.float32)[:, None]
    tangent = (edge_a * uv_b[:, 1:2] - edge_b * uv_a[:, 1:2]) * inv
    bitangent = (edge_b * uv_a[:, 0:1] - edge_a * uv_b[:, 0:1]) * inv
    nv = len(vertices)
    t_sum = np.zeros((nv, 3), np.float64)
    b_sum = np.zeros((nv, 3), np.float64)
    for corner in range(3):
        ids = indices[ok, corner]
        for c in range(3):
            t_sum[:, c] += np.bincount(ids, weights=tangent[ok, c], minlength=nv)
            b_sum[:, c] += np.bincount(ids, weights=bitangent[ok, c], minlength=nv)
    t_sum = t_sum.astype(np.float32)
    b_sum = b_sum.astype(np.float32)
    n = np.asarray(normals, np.float32)
    t = t_sum - n * np.sum(n * t_sum, axis=1, keepdims=True)
    length = np.linalg.norm(t, axis=1)
    weak = length < 1e-8
    if np.any(weak):
        axis = np.where((np.abs(n[weak, 2]) < 0.999)[:, None], np.array([0.0, 0.0, 1.0], np.float32),
                        np.array([0.0, 1.0, 0.0], np.float32))
        t[weak] = np.cross(n[weak], axis)
        length[weak] = np.linalg.norm(t[weak], axis=1)
    t /= np.maximum(length, 1e-8)[:, None]
    hand = np.where(np.sum(np.cross(n, t) * b_sum, axis=1) < 0.0, -1.0, 1.0).astype(np.float32)
    return np.ascontiguousarray(np.column_stack((t, hand)), dtype=np.float32)


def _generate_normals(vertices, indices):
    """Area-weighted vertex normals with identical positions welded, the
    convention of Mesh._generate_normals (scene/_core.py:716-738)."""
    normals = np.zeros_like(vertices)
    if len(indices):
        tri = vertices[indices]
        face = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
        for corner in range(3):
            np.add.at(normals, indices[:, corner], face)
    _unique, groups = np.unique(vertices, axis=0, return_inverse=True)
    groups = groups.reshape(-1)
    welded = np.zeros((len(_unique), 3), dtype=np.float32)
    np.add.at(welded, groups, normals)
    normals = welded[groups]
    lengths = np.linalg.norm(normals, axis=1)
    missing = lengths < 1e-8
    normals[~missing] /= lengths[~missing, None]
    normals[missing] = (0.0, 1.0, 0.0)
    return np.ascontiguousarray(normals, dtype=np.float32)


@dataclass
class Mesh:
    """Placed triangle geometry (scene/_core.py:556-715)."""

    vertices: np.ndarray
    indices: np.ndarray
    material: Material = field(default_factory=Material)
    normals: np.ndarray | None = None
    transform: Transform = field(default_factory=Transform)
    resource: "MeshResource | None" = field(default=None, repr=False)
    visible: bool = True
    name: str | None = None
    metadata: dict = field(default_factory=dict, repr=False)
    deformable: bool = False
    texcoords: np.ndarray | None = field(default=None, repr=False)
    texcoords1: np.ndarray | None = field(default=None, repr=False)
    tangents: np.ndarray | None = field(default=None, repr=False)
    id: int | None = field(default=None, init=False)

    def __post_init__(self):
        if not isinstance(self.visible, bool):
            raise TypeError("visible must be a bool")
        if not isinstance(self.deformable, bool):
            raise TypeError("deformable must be a bool")
        if not isinstance(self.transform, Transform):
            self.transform = Transform(self.transform)
        self.metadata = MappingProxyType(dict(self.metadata))
        if self.resource is not None:
            for name in ("vertices", "indices", "normals", "deformable", "texcoords", "texcoords1", "tangents"):
                setattr(self, name, getattr(self.resource, name))
            return
        self.vertices = np.ascontiguousarray(self.vertices, dtype=np.float32)
        self.indices = np.ascontiguousarray(self.indices, dtype=np.uint32)
        if self.vertices.ndim != 2 or self.vertices.shape[1] != 3:
            raise ValueError("vertices must have shape (vertex_count, 3)")
        if self.indices.ndim != 2 or self.indices.shape[1] != 3:
            raise ValueError("indices must have shape (triangle_count, 3)")
        if self.indices.size and int(self.indices.max()) >= len(self.vertices):
            raise ValueError("an index refers to a vertex that does not exist")
        if self.normals is None:
            self.normals = _generate_normals(self.vertices, self.indices)
        else:
            n = np.ascontiguousarray(self.normals, dtype=np.float32)
            if n.shape != self.vertices.shape:
                raise ValueError("normals must have the same shape as vertices")
            lengths = np.linalg.norm(n, axis=1)
            if np.any(lengths < 1e-8):
                raise ValueError("normals cannot contain zero vectors")
            self.normals = n / lengths[:, None]
        for name in ("texcoords", "texcoords1"):
            value = getattr(self, name)
            if value is None:
                value = np.zeros((len(self.vertices), 2), np.float32)
            value = np.ascontiguousarray(value, dtype=np.float32)
            if value.shape != (len(self.vertices), 2):
                raise ValueError(f"{name} must have shape (vertex_count, 2)")
            setattr(self, name, value)
        if self.tangents is None:
            self.tangents = _generate_tangents(self.vertices, self.indices, self.normals, self.texcoords)
        else:
            t = np.array(self.tangents, dtype=np.float32)
            if t.shape != (len(self.vertices), 4):
                raise ValueError("tangents must have shape (vertex_count, 4)")
            lengths = np.linalg.norm(t[:, :3], axis=1)
            if np.any(lengths < 1e-8):
                raise ValueError("tangent directions cannot contain zero vectors")
            t[:, :3] /= lengths[:, None]
            t[:, 3] = np.where(t[:, 3] < 0.0, -1.0, 1.0)
            self.tangents = t

    @property
    def world_vertices(self):
        linear = self.transform.matrix[:3, :3]
        translation = self.transform.matrix[:3, 3]
        return np.ascontiguousarray(self.vertices @ linear.T + translation, dtype=np.float32)

    @property
    def world_tangents(self):
        """Tangents in world space, orthogonal to the world normals, with the
        handedness flipped by a mirroring transform (scene/_core.py:702-714)."""
        linear = self.transform.matrix[:3, :3]
        directions = self.tangents[:, :3] @ linear.T
        normals = self.world_normals
        directions -= normals * np.sum(directions * normals, axis=1)[:, None]
        directions /= np.linalg.norm(directions, axis=1, keepdims=True)
        handedness = self.tangents[:, 3].copy()
        if np.linalg.det(linear) < 0.0:
            handedness *= -1.0
        return np.ascontiguousarray(np.column_stack((directions, handedness)), dtype=np.float32)

    @property
    def world_normals(self):
        normal_matrix = np.linalg.inv(self.transform.matrix[:3, :3]).T
        result = self.normals @ normal_matrix.T
        result /= np.linalg.norm(result, axis=1, keepdims=True)
        return np.ascontiguousarray(result, dtype=np.float32)


@dataclass
class MeshResource:
    """Reusable object-space geometry shared by instances (scene/_core.py:776-810)."""

    vertices: np.ndarray
    indices: np.ndarray
    material: Material = field(default_factory=Material)
    normals: np.ndarray | None = None
    name: str | None = None
    metadata: dict = field(default_factory=dict, repr=False)
    deformable: bool = False      # positions may change in place (refit instead of rebuild)
    texcoords: np.ndarray | None = field(default=None, repr=False)
    texcoords1: np.ndarray | None = field(default=None, repr=False)
    tangents: np.ndarray | None = field(default=None, repr=False)
    id: int | None = field(default=None, init=False)

    def __post_init__(self):
        if not isinstance(self.deformable, bool):
            raise TypeError("deformable must be a bool")
        checked = Mesh(self.vertices, self.indices, self.material, normals=self.normals, texcoords=self.texcoords,
                       texcoords1=self.texcoords1, tangents=self.tangents)
        for name in ("vertices", "indices", "normals", "texcoords", "texcoords1", "tangents"):
            value = getattr(checked, name)
            value.flags.writeable = False
            setattr(self, name, value)


class Instance(Mesh):
    """A placed occurrence of a MeshResource."""


@dataclass(frozen=True)
class Texture1D:
    """RGBA lookup table with its sampler state (scene/_core.py:137-186): the
    transfer function of a volume.  Three-channel values get an opaque
    alpha."""

    values: np.ndarray = field(compare=False, repr=False)
    address_mode: str = "clamp"
    linear_filter: bool = True

    def __post_init__(self):
        values = np.array(self.values, dtype=np.float32, copy=True)
        if values.ndim != 2 or values.shape[1] not in (3, 4) or len(values) < 1:
            raise ValueError("1D texture values must have shape (length, 3 or 4)")
        if not np.all(np.isfinite(values)):
            raise ValueError("1D texture values must be finite")
        if values.shape[1] == 3:
            values = np.column_stack((values, np.ones(len(values), np.float32)))
        if self.address_mode not in ("clamp", "repeat", "mirror"):
            raise ValueError("address_mode must be clamp, repeat, or mirror")
        values = np.ascontiguousarray(values, np.float32)
        values.flags.writeable = False
        object.__setattr__(self, "values", values)


def _identity_transfer():
    return Texture1D(np.array([[0.0, 0.0, 0.0, 0.0], [1.0, 1.0, 1.0, 1.0]], np.float32))


@dataclass(frozen=True)
class VolumeMaterial:
    """A volume's optical parameters.  The reference's fields
    (scene/_core.py:189-246) drive the reference-compatible emission-
    absorption ray march: the transfer function maps the normalized value to
    emitted RGB and an opacity per ``step_size`` world units, with point-light
    single scattering when ``scattering_scale`` > 0.  ``sigma_t_scale`` and
    ``albedo`` drive the production transport's delta-tracked medium
    (extinction = sigma_t_scale x value; unset, they are density_scale and
    0.9, as for the reference's own material)."""

    sigma_t_scale: float | None = None
    albedo: float | None = None
    transfer_function: Texture1D = field(default_factory=_identity_transfer)
    density_scale: float = 1.0
    emission_scale: float = 1.0
    step_size: float = 0.01
    scattering_scale: float = 0.0
    scattering_color: tuple = (1.0, 1.0, 1.0)
    phase_function: str = "isotropic"
    anisotropy: float = 0.0
    scattering_albedo: tuple = (0.9, 0.9, 0.9)
    scattering_orders: int = 1

    def __post_init__(self):
        if self.sigma_t_scale is not None and not (self.sigma_t_scale >= 0.0 and math.isfinite(self.sigma_t_scale)):
            raise ValueError("sigma_t_scale must be finite and non-negative")
        if self.albedo is not None and not 0.0 <= self.albedo <= 1.0:
            raise ValueError("albedo must be between zero and one")
        if not isinstance(self.transfer_function, Texture1D):
            raise TypeError("transfer_function must be a Texture1D")
        for name in ("density_scale", "emission_scale", "scattering_scale"):
            if not (math.isfinite(getattr(self, name)) and getattr(self, name) >= 0.0):
                raise ValueError(f"{name} must be finite and non-negative")
        if not (math.isfinite(self.step_size) and self.step_size > 0.0):
            raise ValueError("step_size must be positive")
        if self.phase_function not in ("isotropic", "henyey_greenstein"):
            raise ValueError("phase_function must be 'isotropic' or 'henyey_greenstein'")
        if not -0.99 <= self.anisotropy <= 0.99:
            raise ValueError("anisotropy must be between -0.99 and 0.99")
        albedo = _vec3(self.scattering_albedo, "scattering_albedo")
        if np.any(albedo < 0.0) or np.any(albedo > 1.0):
            raise ValueError("scattering_albedo components must be in [0, 1]")
        if np.any(_vec3(self.scattering_color, "scattering_color") < 0.0):
            raise ValueError("scattering_color components cannot be negative")
        if isinstance(self.scattering_orders, bool) or not 1 <= int(self.scattering_orders) <= 8:
            raise ValueError("scattering_orders must be between 1 and 8")


@dataclass
class Volume:
    """Dense scalar field (z, y, x) filling the unit box [0,1]^3 under
    ``transform`` (scene/_core.py:249-400): values are normalized over
    ``value_range`` (linear, log or symlog mapping); with ``missing_data``
    non-finite values are kept as missing; ``clip_planes`` (a, b, c, d) keep
    the points with (a, b, c) . p >= d."""

    data: np.ndarray
    material: VolumeMaterial = field(default_factory=VolumeMaterial)
    transform: Transform = field(default_factory=Transform)
    value_range: tuple | None = None
    value_mapping: str = "linear"
    linear_threshold: float = 1.0
    missing_data: bool = False
    clip_planes: tuple = ()
    visible: bool = True
    name: str | None = None
    id: int | None = field(default=None, init=False)

    def __post_init__(self):
        d = np.array(self.data, dtype=np.float32, copy=True, order="C")
        if d.ndim != 3 or min(d.shape) < 2:
            raise ValueError("volume data must have shape (depth, height, width) with dimensions >= 2")
        if self.missing_data:
            d[~np.isfinite(d)] = np.nan
        elif not np.all(np.isfinite(d)):
            raise ValueError("volume data must contain finite values")
        d.flags.writeable = False
        self.data = d
        if self.value_mapping not in ("linear", "log", "symlog"):
            raise ValueError("value_mapping must be 'linear', 'log' or 'symlog'")
        if self.value_range is None:
            finite = d[np.isfinite(d)]
            if not finite.size:
                raise ValueError("volume data must contain at least one finite value")
            lo, hi = float(finite.min()), float(finite.max())
            self.value_range = (min(0.0, lo), max(1.0, lo)) if lo == hi else (lo, hi)
        else:
            self.value_range = tuple(float(v) for v in self.value_range)
            if len(self.value_range) != 2 or not self.value_range[0] < self.value_range[1]:
                raise ValueError("value_range must be two increasing values")
        self.clip_planes = tuple(tuple(float(c) for c in plane) for plane in self.clip_planes)
        if any(len(plane) != 4 for plane in self.clip_planes) or len(self.clip_planes) > 8:
            raise ValueError("clip_planes must hold at most eight (a, b, c, d) planes")
        if not isinstance(self.transform, Transform):
            self.transform = Transform(self.transform)

    @property
    def shape(self):
        return self.data.shape

    @property
    def normalized_data(self):
        """Values mapped to [0, 1] over value_range (missing values NaN when
        missing_data, else 0), as the reference normalizes them."""
        low, high = self.value_range
        with np.errstate(divide="ignore", invalid="ignore"):
            if self.value_mapping == "log":
                normalized = (np.log(self.data) - np.log(low)) / (np.log(high) - np.log(low))
            elif self.value_mapping == "symlog":
                f = lambda v: np.sign(v) * np.log1p(np.abs(v) / self.linear_threshold)  # noqa: E731
                normalized = (f(self.data) - f(low)) / (f(high) - f(low))
            else:
                normalized = (self.data - low) / (high - low)
        return np.ascontiguousarray(np.where(np.isfinite(normalized), np.clip(normalized, 0.0, 1.0),
                                             np.nan if self.missing_data else 0.0))


class Scene:
    """Scene container with stable ids and revision counters
    (scene/_core.py:943-3093)."""

    def __init__(self, meshes=(), lights=(), mesh_resources=(), volumes=(), environment=None, metadata=None):
        self.meshes = []
        self.lights = []
        self.mesh_resources = []
        self.volumes = []
        self.environment = None
        self.metadata = dict(metadata or {})
        self._revision = 0
        self._geometry_revision = 0
        self._shading_revision = 0
        self._transform_revision = 0
        self._next_resource_id = 1
        self._next_mesh_resource_id = 1
        self._next_material_id = 1
        self._material_ids = {}
        for resource in mesh_resources:
            self._attach_mesh_resource(resource)
            self.mesh_resources.append(resource)
        for mesh in meshes:
            if not isinstance(mesh, Mesh):
                raise TypeError("scene resources must be mesh or light objects")
            self._attach(mesh)
            self._register_material(mesh.material)
            self.meshes.append(mesh)
        for light in lights:
            self.add_light(light)
        for volume in volumes:
            self._attach(volume)
            self.volumes.append(volume)
        if environment is not None:
            self.set_environment(environment)

    # -- identity and revisions -------------------------------------------
    @property
    def revision(self):
        return self._revision

    @property
    def geometry_revision(self):
        return self._geometry_revision

    @property
    def shading_revision(self):
        return self._shading_revision

    @property
    def transform_revision(self):
        return self._transform_revision

    def _changed(self, *, geometry=False, shading=False, transform=False):
        self._revision += 1
        self._geometry_revision += int(geometry)
        self._shading_revision += int(shading)
        self._transform_revision += int(transform)

    def _attach(self, resource):
        if resource.id is not None:
            raise ValueError("a scene resource cannot belong to multiple scenes")
        resource.id = self._next_resource_id
        self._next_resource_id += 1

    def _attach_mesh_resource(self, resource):
        if resource.id is not None:
            raise ValueError("a mesh resource cannot belong to multiple scenes")
        resource.id = self._next_mesh_resource_id
        self._next_mesh_resource_id += 1

    def _register_material(self, material):
        existing = self._material_ids.get(id(material))
        if existing is not None and existing[0] is material:
            return existing[1]
        material_id = self._next_material_id
        self._next_material_id += 1
        self._material_ids[id(material)] = (material, material_id)
        return material_id

    def material_id(self, material):
        existing = self._material_ids.get(id(material))
        if existing is None or existing[0] is not material:
            raise KeyError("material is not attached to this scene")
        return existing[1]

    # -- membership -------------------------------------------------------
    @property
    def instances(self):
        return tuple(self.meshes)

    @property
    def visible_meshes(self):
        return tuple(mesh for mesh in self.meshes if mesh.visible)

    @property
    def visible_volumes(self):
        return tuple(volume for volume in self.volumes if volume.visible)

    def create_mesh(self, vertices, indices, material=None, *, normals=None, name=None, metadata=None,
                    deformable=False, texcoords=None, texcoords1=None, tangents=None):
        resource = MeshResource(vertices, indices, material or Material(), normals=normals, name=name,
                                metadata={} if metadata is None else metadata, deformable=deformable,
                                texcoords=texcoords, texcoords1=texcoords1, tangents=tangents)
        self._attach_mesh_resource(resource)
        self.mesh_resources.append(resource)
        return resource

    create_mesh_resource = create_mesh

    def add_mesh(self, vertices, indices, material=None, *, normals=None, transform=None, name=None,
                 metadata=None, deformable=False, texcoords=None, texcoords1=None, tangents=None):
        resource = self.create_mesh(vertices, indices, material, normals=normals, name=name, metadata=metadata,
                                    deformable=deformable, texcoords=texcoords, texcoords1=texcoords1,
                                    tangents=tangents)
        return self.add_instance(resource, transform=transform, name=name, metadata=metadata)

    def _resolve_resource(self, resource):
        for candidate in self.mesh_resources:
            if candidate is resource or candidate.id == resource:
                return candidate
        raise KeyError("mesh resource is not part of this scene")

    def add_instance(self, resource, *, transform=None, material=None, visible=True, name=None, metadata=None):
        resource = self._resolve_resource(resource)
        instance = Instance(resource.vertices, resource.indices,
                            resource.material if material is None else material,
                            transform=Transform() if transform is None else transform,
                            resource=resource, visible=visible, name=name,
                            metadata={} if metadata is None else metadata)
        self._attach(instance)
        self._register_material(instance.material)
        self.meshes.append(instance)
        self._changed(geometry=True, shading=True)
        return instance

    def add_instances(self, resource, transforms, *, materials=None, visible=True, names=None):
        resource = self._resolve_resource(resource)
        transforms = [t if isinstance(t, Transform) else Transform(t) for t in transforms]
        count = len(transforms)
        if materials is None:
            materials = [resource.material] * count
        elif isinstance(materials, Material):
            materials = [materials] * count
        else:
            materials = list(materials)
            if len(materials) != count:
                raise ValueError(f"expected {count} materials, got {len(materials)}")
        names = [names] * count if names is None or isinstance(names, str) else list(names)
        created = []
        for transform, material, name in zip(transforms, materials, names):
            instance = Instance(resource.vertices, resource.indices, material, transform=transform,
                                resource=resource, visible=visible, name=name)
            self._attach(instance)
            self._register_material(material)
            self.meshes.append(instance)
            created.append(instance)
        if created:
            self._changed(geometry=True, shading=True)
        return tuple(created)

    def update_mesh_resource(self, resource, *, vertices=None, indices=None, normals=None, material=None):
        """Replace shared geometry or its default material and synchronise
        every instance of it (scene/_core.py:1579-1636).  New positions or
        topology without new normals regenerate the normals."""
        resource = self._resolve_resource(resource)
        geometry = vertices is not None or indices is not None
        if normals is None and not geometry:
            normals = resource.normals
        old_material = resource.material
        candidate = MeshResource(resource.vertices if vertices is None else vertices,
                                 resource.indices if indices is None else indices,
                                 resource.material if material is None else material,
                                 normals=normals, deformable=resource.deformable)
        resource.vertices, resource.indices, resource.normals = candidate.vertices, candidate.indices, candidate.normals
        resource.material = candidate.material
        for instance in self.meshes:
            if instance.resource is not resource:
                continue
            instance.vertices, instance.indices, instance.normals = (candidate.vertices, candidate.indices,
                                                                     candidate.normals)
            if material is not None and instance.material is old_material:
                instance.material = candidate.material
        self._register_material(candidate.material)
        self._changed(geometry=geometry, shading=geometry or material is not None or normals is not None)
        return resource

    def update_instance_transforms(self, instances, transforms):
        """New transforms for several instances, one revision step
        (scene/_core.py:1809-1811)."""
        instances, transforms = list(instances), list(transforms)
        if len(instances) != len(transforms):
            raise ValueError("instances and transforms must have the same length")
        for instance, transform in zip(instances, transforms):
            instance.transform = transform if isinstance(transform, Transform) else Transform(transform)
        if instances:
            self._changed(transform=True)
        return tuple(instances)

    def update_instance(self, instance, *, transform=None, material=None, visible=None):
        if transform is not None:
            instance.transform = transform if isinstance(transform, Transform) else Transform(transform)
        if material is not None:
            instance.material = material
            self._register_material(material)
        if visible is not None:
            instance.visible = bool(visible)
        self._changed(geometry=visible is not None, shading=material is not None, transform=transform is not None)
        return instance

    def add_light(self, light):
        if not isinstance(light, LIGHT_TYPES):
            raise TypeError("light must be a PointLight, DirectionalLight, or SpotLight")
        self._attach(light)
        self.lights.append(light)
        self._changed(shading=True)
        return light

    def add_point_light(self, position, color=(1.0, 1.0, 1.0), intensity=1.0, *, range=None):
        return self.add_light(PointLight(position, color, intensity, range))

    def add_directional_light(self, direction, color=(1.0, 1.0, 1.0), intensity=1.0):
        return self.add_light(DirectionalLight(direction, color, intensity))

    def set_environment(self, environment=None, **parameters):
        if environment is not None and parameters:
            raise TypeError("pass an EnvironmentLight or keyword parameters, not both")
        if parameters:
            environment = EnvironmentLight(**parameters)
        if environment is not None and not isinstance(environment, EnvironmentLight):
            raise TypeError("environment must be an EnvironmentLight or None")
        if environment is self.environment:
            return environment
        self.environment = environment
        self._changed(shading=True)
        return environment

    def add_volume(self, data, material=None, *, transform=None, value_range=None, value_mapping="linear",
                   linear_threshold=1.0, missing_data=False, clip_planes=(), visible=True, name=None):
        volume = Volume(data, material or VolumeMaterial(), Transform() if transform is None else transform,
                        value_range=value_range, value_mapping=value_mapping, linear_threshold=linear_threshold,
                        missing_data=missing_data, clip_planes=clip_planes, visible=visible, name=name)
        self._attach(volume)
        self.volumes.append(volume)
        self._changed(geometry=True, shading=True)
        return volume

    # -- packing helpers (same layouts as the reference) -----------------
    def triangles(self):
        """World-space triangle soup, colours and emissions in packed order
        (Scene.triangles, scene/_core.py:2732-2753)."""
        tris, colors, emissions = [], [], []
        for mesh in self.visible_meshes:
            t = mesh.world_vertices[mesh.indices]
            tris.append(t)
            colors.extend([mesh.material.base_color] * len(t))
            emissions.extend([mesh.material.emission] * len(t))
        if not tris:
            return (np.empty((0, 3, 3), np.float32), np.empty((0, 3), np.float32), np.empty((0, 3), np.float32))
        return (np.concatenate(tris), np.asarray(colors, dtype=np.float32).reshape(-1, 3),
                np.asarray(emissions, dtype=np.float32).reshape(-1, 3))

    def triangle_instance_ids(self):
        values = [np.full(len(m.indices), m.id, np.uint32) for m in self.visible_meshes if len(m.indices)]
        return np.concatenate(values) if values else np.empty(0, np.uint32)

    @property
    def emissive_light_weight(self):
        total = 0.0
        for mesh in self.visible_meshes:
            lum = float(np.dot(np.asarray(mesh.material.emission, np.float64), _LUMINANCE))
            if lum <= 0.0:
                continue
            t = mesh.world_vertices[mesh.indices]
            areas = 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1)
            total += float(areas[areas > 1e-12].sum()) * lum
        return total

    @property
    def bounds(self):
        tris = self.triangles()[0]
        if not len(tris):
            return None
        flat = tris.reshape(-1, 3)
        return flat.min(axis=0), flat.max(axis=0)
