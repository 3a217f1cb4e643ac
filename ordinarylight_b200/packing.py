"""Scene and camera packing for the C ABI.

Works on any object with the reference's scene surface (``visible_meshes``,
mesh ``vertices``/``indices``/``normals``/``transform``/``material``/
``resource``/``id``, ``lights``, ``environment``, ``visible_volumes``), so the
reference's ``ordinarylight.Scene`` and this package's mirror both pack.

Geometry stays indexed in object space: one bottom-level mesh per distinct
``MeshResource`` (or per resource-less ``Mesh``), one instance per visible
mesh with triangles, in ``visible_meshes`` order.  The instance's packed
primitive base is the running triangle count in that order, so the
device-reported primitive index equals the index into ``Scene.triangles()``
(ordinarylight/scene/_core.py:2732-2753) that the CPU reference reports.
"""

from __future__ import annotations

from dataclasses import dataclass, fields
import math

import numpy as np

from . import _native

_LUMINANCE = np.array((0.2126, 0.7152, 0.0722), np.float64)


@dataclass
class PackedScene:
    mesh_vertex_offset: np.ndarray
    mesh_triangle_offset: np.ndarray
    vertices: np.ndarray
    normals: np.ndarray
    indices: np.ndarray
    instance_object_to_world: np.ndarray
    instance_mesh: np.ndarray
    instance_material: np.ndarray
    instance_id: np.ndarray
    instance_primitive_offset: np.ndarray
    materials: np.ndarray
    emitters: np.ndarray
    emissive_weight: float
    lights: np.ndarray
    environment_kind: int
    environment_color: tuple
    environment_rotation: float
    environment_image: np.ndarray | None
    volume: dict | None
    total_triangles: int
    mesh_sources: tuple = ()      # the MeshResource (or Mesh) behind each packed mesh
    # textures (texture_bindings empty: an untextured scene)
    texcoords: np.ndarray | None = None          # [total_vertices, 4] uv0, uv1
    tangents: np.ndarray | None = None           # [total_vertices, 4] object-space xyz, handedness
    texture_words: np.ndarray | None = None      # Scene.texture_data layout
    texture_bindings: np.ndarray | None = None   # [n, 8]
    material_textures: np.ndarray | None = None  # [num_materials, 12]
    # volumes in the reference's model (records [n, 72], grids, luts [m, 4])
    ref_volumes: dict | None = None
    volume_count: int = 0          # visible volumes of the scene

    def descriptor(self) -> _native.OlcSceneDesc:
        d = _native.OlcSceneDesc()
        f32, u32 = _native.c_float, _native.c_uint32
        d.num_meshes = len(self.mesh_vertex_offset) - 1
        d.mesh_vertex_offset = _native.typed_ptr(self.mesh_vertex_offset, u32)
        d.mesh_triangle_offset = _native.typed_ptr(self.mesh_triangle_offset, u32)
        d.vertices = _native.typed_ptr(self.vertices, f32)
        d.normals = _native.typed_ptr(self.normals, f32)
        d.indices = _native.typed_ptr(self.indices, u32)
        d.num_instances = len(self.instance_mesh)
        d.instance_object_to_world = _native.typed_ptr(self.instance_object_to_world, f32)
        d.instance_mesh = _native.typed_ptr(self.instance_mesh, u32)
        d.instance_material = _native.typed_ptr(self.instance_material, u32)
        d.instance_id = _native.typed_ptr(self.instance_id, u32)
        d.instance_primitive_offset = _native.typed_ptr(self.instance_primitive_offset, u32)
        d.num_materials = len(self.materials)
        d.materials = _native.typed_ptr(self.materials, f32)
        d.num_emitters = len(self.emitters)
        d.emitters = _native.typed_ptr(self.emitters if len(self.emitters) else None, f32)
        d.emissive_weight = float(self.emissive_weight)
        d.num_lights = len(self.lights)
        d.lights = _native.typed_ptr(self.lights if len(self.lights) else None, f32)
        d.environment_kind = self.environment_kind
        for k in range(3):
            d.environment_color[k] = float(self.environment_color[k])
        d.environment_rotation = float(self.environment_rotation)
        if self.environment_image is not None:
            d.environment_height, d.environment_width = self.environment_image.shape[:2]
            d.environment_image = _native.typed_ptr(self.environment_image, f32)
        if self.volume is not None:
            v = self.volume
            d.volume_present = 1
            nz, ny, nx = v["density"].shape
            d.volume_dims[0], d.volume_dims[1], d.volume_dims[2] = nx, ny, nz
            d.volume_density = _native.typed_ptr(v["density"], f32)
            for k in range(12):
                d.volume_world_to_box[k] = float(v["world_to_box"].reshape(-1)[k])
            d.volume_sigma_t_scale = float(v["sigma_t_scale"])
            d.volume_albedo = float(v["albedo"])
            d.volume_max_density = float(v["max_density"])
        if self.ref_volumes is not None:
            rv = self.ref_volumes
            d.num_ref_volumes = len(rv["records"])
            d.ref_volume_records = _native.typed_ptr(rv["records"], f32)
            d.ref_grid_values = len(rv["grids"])
            d.ref_volume_grids = _native.typed_ptr(rv["grids"], f32)
            d.ref_lut_entries = len(rv["luts"])
            d.ref_volume_luts = _native.typed_ptr(rv["luts"], f32)
        if self.texture_bindings is not None and len(self.texture_bindings):
            d.texcoords = _native.typed_ptr(self.texcoords, f32)
            d.tangents = _native.typed_ptr(self.tangents, f32)
            d.num_texture_words = len(self.texture_words)
            d.texture_words = _native.typed_ptr(self.texture_words, u32)
            d.num_texture_bindings = len(self.texture_bindings)
            d.texture_bindings = _native.typed_ptr(self.texture_bindings, f32)
            d.material_textures = _native.typed_ptr(self.material_textures, f32)
        return d

    # -- files -------------------------------------------------------------
    _DICT_FIELDS = ("volume", "ref_volumes")

    def save(self, path) -> None:
        """Write the packed arrays to an .npz file (the mesh source objects
        are not kept): a scene packed where its objects exist, rendered
        elsewhere."""
        out = {}
        for f in fields(self):
            value = getattr(self, f.name)
            if f.name == "mesh_sources":
                continue
            if f.name in self._DICT_FIELDS:
                out[f"{f.name}__present"] = np.array(value is not None)
                for k, v in (value or {}).items():
                    out[f"{f.name}__{k}"] = np.asarray(v)
            elif value is None:
                out[f"{f.name}__none"] = np.array(True)
            else:
                out[f.name] = np.asarray(value)
        np.savez_compressed(path, **out)

    @classmethod
    def load(cls, path) -> "PackedScene":
        data = np.load(path, allow_pickle=False)
        values = {}
        for f in fields(cls):
            if f.name == "mesh_sources":
                continue
            if f.name in cls._DICT_FIELDS:
                if bool(data[f"{f.name}__present"]):
                    prefix = f"{f.name}__"
                    values[f.name] = {k[len(prefix):]: (data[k][()] if data[k].ndim == 0 else data[k])
                                      for k in data.files if k.startswith(prefix) and k != f"{f.name}__present"}
                else:
                    values[f.name] = None
            elif f"{f.name}__none" in data.files:
                values[f.name] = None
            else:
                v = data[f.name]
                values[f.name] = v[()] if v.ndim == 0 else v
        values["environment_color"] = tuple(float(c) for c in values["environment_color"])
        for name in ("emissive_weight", "environment_rotation"):
            values[name] = float(values[name])
        for name in ("environment_kind", "total_triangles", "volume_count"):
            values[name] = int(values[name])
        return cls(**values)


def _material_record(material, material_id: int) -> np.ndarray:
    rec = np.zeros(16, np.float32)
    rec[0:3] = np.asarray(material.base_color, np.float32)
    rec[3] = float(getattr(material, "roughness", 1.0))
    rec[4:7] = np.asarray(material.emission, np.float32)
    rec[7] = float(getattr(material, "metallic", 0.0))
    rec[8] = 1.0 if getattr(material, "emission_two_sided", False) else 0.0
    rec[9] = np.array([material_id], np.uint32).view(np.float32)[0]
    rec[10] = float(getattr(material, "transmission", 0.0))
    rec[11] = float(getattr(material, "ior", 1.5))
    return rec


# -- textures ---------------------------------------------------------------
TEXTURE_SLOTS = ("base_color", "metallic_roughness", "emissive", "normal", "occlusion", "transmission")
_WRAP_CODES = {"repeat": 0, "clamp": 1, "mirror": 2}


def texture_mips(pixels, *, srgb):
    """RGBA8 mip pyramid down to 1x1: 2x2 box filter of edge-padded levels,
    averaged in linear space for sRGB data and re-encoded per level
    (Scene._texture_mips, scene/_core.py:3045-3077)."""
    current = np.asarray(pixels, dtype=np.float32) / 255.0
    if srgb:
        rgb = current[..., :3]
        current[..., :3] = np.where(rgb <= 0.04045, rgb / 12.92, ((rgb + 0.055) / 1.055) ** 2.4)
    levels = []
    while True:
        encoded = current.copy()
        if srgb:
            rgb = np.maximum(encoded[..., :3], 0.0)
            encoded[..., :3] = np.where(rgb <= 0.0031308, rgb * 12.92, 1.055 * rgb ** (1.0 / 2.4) - 0.055)
        levels.append(np.clip(encoded * 255.0 + 0.5, 0, 255).astype(np.uint8))
        height, width, _ = current.shape
        if width == 1 and height == 1:
            return levels
        nw, nh = max(1, (width + 1) // 2), max(1, (height + 1) // 2)
        padded = np.pad(current, ((0, height & 1), (0, width & 1), (0, 0)), mode="edge")
        current = padded.reshape(nh, 2, nw, 2, 4).mean(axis=(1, 3))


def texture_words(textures):
    """Header (count, then 8 words per texture: sRGB offset, linear offset,
    width, height, wrap/filter flags, levels, 0, 0) followed by each
    texture's sRGB and linear RGBA8 pyramids (Scene.texture_data,
    scene/_core.py:3005-3043)."""
    header = np.zeros(1 + 8 * len(textures), np.uint32)
    header[0] = len(textures)
    chunks, offset = [header], len(header)
    for index, texture in enumerate(textures):
        height, width, _ = texture.pixels.shape
        flags = _WRAP_CODES[texture.wrap_s] | (_WRAP_CODES[texture.wrap_t] << 2) | (int(texture.linear_filter) << 4)
        words = []
        for srgb in (True, False):
            levels = texture_mips(texture.pixels, srgb=srgb)
            words.append(np.concatenate([lv.reshape(-1, 4).copy().view(np.uint32).reshape(-1) for lv in levels]))
        header[1 + 8 * index:9 + 8 * index] = (offset, offset + len(words[0]), width, height, flags, len(levels), 0, 0)
        chunks += words
        offset += len(words[0]) + len(words[1])
    return np.ascontiguousarray(np.concatenate(chunks), dtype=np.uint32)


def _texture_tables(meshes, materials_in_order):
    """Textures in first-use order, (texture, transform) bindings and the
    per-material binding records (Scene.textures / texture_bindings /
    texture_binding_data, scene/_core.py:2928-3003)."""
    textures, bindings = [], []
    for mesh in meshes:
        material = mesh.material
        for slot in TEXTURE_SLOTS:
            texture = getattr(material, f"{slot}_texture", None)
            if texture is None:
                continue
            transform = getattr(material, f"{slot}_transform")
            if all(texture is not t for t in textures):
                textures.append(texture)
            if all(texture is not t or transform != tf for t, tf in bindings):
                bindings.append((texture, transform))
    if not bindings:
        return None
    records = np.zeros((len(bindings), 8), np.float32)
    for k, (texture, transform) in enumerate(bindings):
        index = next(i for i, t in enumerate(textures) if t is texture)
        records[k] = (index, np.cos(transform.rotation), np.sin(transform.rotation), transform.texcoord_set,
                      *transform.offset, *transform.scale)
    mat = np.zeros((len(materials_in_order), 12), np.float32)
    for m, material in enumerate(materials_in_order):
        uses_uv1 = 0.0
        for k, slot in enumerate(TEXTURE_SLOTS):
            texture = getattr(material, f"{slot}_texture", None)
            transform = getattr(material, f"{slot}_transform", None)
            mat[m, k] = next((i for i, (t, tf) in enumerate(bindings) if t is texture and tf == transform), -1)
            if texture is not None and transform.texcoord_set == 1:
                uses_uv1 = 1.0
        mat[m, 6] = float(getattr(material, "normal_scale", 1.0))
        mat[m, 7] = float(getattr(material, "occlusion_strength", 1.0))
        mat[m, 8] = uses_uv1
    return texture_words(textures), records, mat


def emitter_records(scene):
    """Emissive triangles with a power CDF: the records and probabilities of
    Scene.emissive_triangle_data (scene/_core.py:2637-2691), computed with
    array operations.  Returns (records [n, 20] float32, total weight)."""
    chunks, weights, sided = [], [], []
    for mesh in scene.visible_meshes:
        emission = np.asarray(mesh.material.emission, np.float32)
        if not np.any(emission > 0.0) or not len(mesh.indices):
            continue
        tris = mesh.world_vertices[mesh.indices]
        area = 0.5 * np.linalg.norm(np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0]), axis=1)
        keep = area > 1e-12
        if not np.any(keep):
            continue
        tris, area = tris[keep], area[keep]
        rec = np.zeros((len(tris), 20), np.float32)
        rec[:, 0:3] = tris[:, 0]
        rec[:, 4:7] = tris[:, 1]
        rec[:, 8:11] = tris[:, 2]
        rec[:, 12:15] = emission
        rec[:, 15] = area
        chunks.append(rec)
        weights.append(area.astype(np.float64) * float(np.dot(emission.astype(np.float64), _LUMINANCE)))
        sided.append(np.full(len(tris), 1.0 if getattr(mesh.material, "emission_two_sided", False) else 0.0,
                             np.float32))
    if not chunks:
        return np.zeros((0, 20), np.float32), 0.0
    rec = np.concatenate(chunks)
    w = np.concatenate(weights)
    total = float(w.sum())
    prob = w / total if total > 0.0 else np.full(len(w), 1.0 / len(w))
    cdf = np.cumsum(prob)
    cdf[-1] = 1.0
    rec[:, 16] = cdf.astype(np.float32)
    rec[:, 17] = prob.astype(np.float32)
    rec[:, 18] = np.concatenate(sided)
    return rec, float(scene.emissive_light_weight) if hasattr(scene, "emissive_light_weight") else total


def light_records(scene) -> np.ndarray:
    """Analytic lights in the layout of Scene.analytic_light_data
    (scene/_core.py:2578-2632), without the environment record."""
    records = []
    for light in getattr(scene, "lights", ()):
        name = type(light).__name__
        rec = np.zeros((4, 4), np.float32)
        rec[2, :3] = np.asarray(light.color, np.float32)
        rec[2, 3] = float(light.intensity)
        if name == "PointLight":
            rec[0, :3] = np.asarray(light.position, np.float32)
            rec[0, 3] = 0.0
            rec[1, 3] = float(light.range or 0.0)
        elif name == "DirectionalLight":
            direction = np.asarray(light.direction, np.float32)
            rec[0, 3] = 1.0
            rec[1, :3] = direction / np.linalg.norm(direction)
        elif name == "SpotLight":
            direction = np.asarray(light.direction, np.float32)
            rec[0, :3] = np.asarray(light.position, np.float32)
            rec[0, 3] = 2.0
            rec[1, :3] = direction / np.linalg.norm(direction)
            rec[1, 3] = float(light.range or 0.0)
            rec[3, 0] = math.cos(light.inner_cone_angle)
            rec[3, 1] = math.cos(light.outer_cone_angle)
        else:
            raise TypeError(f"unsupported light type {name}")
        records.append(rec.reshape(-1))
    if not records:
        return np.zeros((0, 16), np.float32)
    return np.ascontiguousarray(np.stack(records), np.float32)


def _volume_record(scene):
    volumes = tuple(getattr(scene, "visible_volumes", ()))
    if not volumes:
        return None
    if len(volumes) > 1:
        return None   # the production medium is one grid; the renderer refuses such scenes in production mode
    vol = volumes[0]
    density = np.ascontiguousarray(getattr(vol, "data", None), np.float32)
    if density.ndim != 3:
        raise RuntimeError("volume data must be a dense 3D grid")
    material = getattr(vol, "material", None)
    sigma = getattr(material, "sigma_t_scale", None)
    if sigma is None:
        sigma = getattr(material, "density_scale", 1.0)
    albedo = getattr(material, "albedo", None)
    sigma, albedo = float(sigma), 0.9 if albedo is None else float(albedo)
    w2b = np.linalg.inv(np.asarray(vol.transform.matrix, np.float64))[:3, :4].astype(np.float32)
    return {"density": density, "world_to_box": w2b, "sigma_t_scale": sigma, "albedo": albedo,
            "max_density": float(density.max()) if density.size else 0.0}


_ADDRESS = {"clamp": 0, "repeat": 1, "mirror": 2}


def _ref_volume_tables(scene):
    """Visible volumes in the reference's model for the reference-compatible
    ray march (olc_scene_desc's 72-float records): the inverse transform, the
    normalized grid (Volume.normalized_data), the transfer function and the
    optical parameters (ordinarylight/volume/_core.py:252-504)."""
    volumes = tuple(getattr(scene, "visible_volumes", ()))
    if not volumes:
        return None
    if any(getattr(v.material, "transfer_function", None) is None for v in volumes):
        return None   # volumes without the reference's optical model
    if len(volumes) > 8:
        raise ValueError("the reference-compatible mode integrates at most 8 visible volumes per scene")
    records, grids, luts = [], [], []
    grid_off = lut_off = 0
    for vol in volumes:
        m = vol.material
        tf = m.transfer_function
        grid = np.ascontiguousarray(vol.normalized_data, np.float32)
        nz, ny, nx = grid.shape
        lut = np.ascontiguousarray(tf.values, np.float32).reshape(-1, 4)
        planes = [tuple(map(float, p)) for p in getattr(vol, "clip_planes", ())]
        if len(planes) > 8:
            raise ValueError("a volume has at most 8 clip planes")
        rec = np.zeros(72, np.float32)
        ints = rec.view(np.uint32)
        rec[0:12] = np.linalg.inv(np.asarray(vol.transform.matrix, np.float64)).astype(np.float32)[:3, :4].reshape(-1)
        ints[12:16] = (nx, ny, nz, len(lut))
        ints[16:24] = (grid_off, lut_off, _ADDRESS[tf.address_mode], int(bool(tf.linear_filter)),
                       int(bool(getattr(vol, "missing_data", False))), len(planes),
                       int(m.phase_function == "henyey_greenstein"), int(m.scattering_orders))
        rec[24:28] = (m.density_scale, m.emission_scale, m.step_size, m.scattering_scale)
        rec[28:31] = m.scattering_color
        rec[31] = m.anisotropy
        rec[32:35] = m.scattering_albedo
        for k, plane in enumerate(planes):
            rec[36 + 4 * k:40 + 4 * k] = plane
        records.append(rec)
        grids.append(grid.reshape(-1))
        luts.append(lut)
        grid_off += grid.size
        lut_off += len(lut)
    return {"records": np.ascontiguousarray(np.stack(records)), "grids": np.ascontiguousarray(np.concatenate(grids)),
            "luts": np.ascontiguousarray(np.concatenate(luts))}


def pack_scene(scene) -> PackedScene:
    """Flatten a scene into the arrays of olc_scene_desc."""
    mesh_index = {}
    sources = []
    vertices, normals, indices, texcoords, tangents = [], [], [], [], []
    material_objects = []
    v_off, t_off = [0], [0]
    inst_xf, inst_mesh, inst_mat, inst_id, inst_prim = [], [], [], [], []
    materials, material_index = [], {}
    prim = 0
    material_id = getattr(scene, "material_id", None)
    for mesh in scene.visible_meshes:
        count = len(mesh.indices)
        if count == 0:
            continue
        key = id(mesh.resource) if getattr(mesh, "resource", None) is not None else id(mesh)
        if key not in mesh_index:
            mesh_index[key] = len(v_off) - 1
            sources.append(mesh.resource if getattr(mesh, "resource", None) is not None else mesh)
            verts = np.ascontiguousarray(mesh.vertices, np.float32).reshape(-1, 3)
            vertices.append(verts)
            n = getattr(mesh, "normals", None)
            normals.append(np.ascontiguousarray(n if n is not None else np.zeros_like(verts), np.float32))
            indices.append(np.ascontiguousarray(mesh.indices, np.uint32).reshape(-1, 3))
            uv0 = getattr(mesh, "texcoords", None)
            uv1 = getattr(mesh, "texcoords1", None)
            tan = getattr(mesh, "tangents", None)
            zeros2 = np.zeros((len(verts), 2), np.float32)
            texcoords.append(np.column_stack((zeros2 if uv0 is None else np.asarray(uv0, np.float32),
                                              zeros2 if uv1 is None else np.asarray(uv1, np.float32))))
            tangents.append(np.tile(np.array([1.0, 0.0, 0.0, 1.0], np.float32), (len(verts), 1)) if tan is None
                            else np.asarray(tan, np.float32).reshape(-1, 4))
            v_off.append(v_off[-1] + len(verts))
            t_off.append(t_off[-1] + len(mesh.indices))
        mat = mesh.material
        if id(mat) not in material_index:
            mid = 0
            if callable(material_id):
                try:
                    mid = int(material_id(mat))
                except KeyError:
                    mid = 0
            material_index[id(mat)] = len(materials)
            materials.append(_material_record(mat, mid))
            material_objects.append(mat)
        inst_xf.append(np.asarray(mesh.transform.matrix, np.float32)[:3, :4].reshape(-1))
        inst_mesh.append(mesh_index[id(mesh.resource) if getattr(mesh, "resource", None) is not None else id(mesh)])
        inst_mat.append(material_index[id(mat)])
        inst_id.append(int(mesh.id) if mesh.id is not None else 0)
        inst_prim.append(prim)
        prim += count
    emitters, weight = emitter_records(scene)
    env = getattr(scene, "environment", None)
    env_kind, env_color, env_rot, env_img = _native.ENV_NONE, (0.0, 0.0, 0.0), 0.0, None
    if env is not None:
        env_color = tuple(float(c) * float(env.intensity) for c in env.color)
        env_rot = float(env.rotation)
        if getattr(env, "image", None) is not None:
            env_kind = _native.ENV_EQUIRECT
            env_img = np.ascontiguousarray(np.asarray(env.image, np.float32)[..., :3])
        else:
            env_kind = _native.ENV_CONSTANT

    def stack(parts, dtype, shape):
        return np.ascontiguousarray(np.concatenate(parts), dtype) if parts else np.zeros(shape, dtype)

    tables = _texture_tables([m for m in scene.visible_meshes if len(m.indices)], material_objects)
    tex = {}
    if tables is not None:
        tex = dict(texcoords=stack(texcoords, np.float32, (0, 4)), tangents=stack(tangents, np.float32, (0, 4)),
                   texture_words=tables[0], texture_bindings=tables[1], material_textures=tables[2])

    return PackedScene(
        mesh_vertex_offset=np.asarray(v_off, np.uint32),
        mesh_triangle_offset=np.asarray(t_off, np.uint32),
        vertices=stack(vertices, np.float32, (0, 3)),
        normals=stack(normals, np.float32, (0, 3)),
        indices=stack(indices, np.uint32, (0, 3)),
        instance_object_to_world=np.ascontiguousarray(np.asarray(inst_xf, np.float32).reshape(-1, 12)),
        instance_mesh=np.asarray(inst_mesh, np.uint32),
        instance_material=np.asarray(inst_mat, np.uint32),
        instance_id=np.asarray(inst_id, np.uint32),
        instance_primitive_offset=np.asarray(inst_prim, np.uint32),
        materials=np.ascontiguousarray(np.asarray(materials, np.float32).reshape(-1, 16)),
        emitters=np.ascontiguousarray(emitters),
        emissive_weight=weight,
        lights=light_records(scene),
        environment_kind=env_kind,
        environment_color=env_color,
        environment_rotation=env_rot,
        environment_image=env_img,
        volume=_volume_record(scene),
        ref_volumes=_ref_volume_tables(scene),
        volume_count=len(tuple(getattr(scene, "visible_volumes", ()))),
        total_triangles=prim,
        mesh_sources=tuple(sources),
        **tex,
    )


def refit_mask(old: PackedScene, new: PackedScene):
    """Meshes to refit when ``new`` replaces ``old`` in place, or None when
    the scene must be uploaded again.  The rules of the reference's in-place
    update (_try_update_window_scene, ordinarylight/targets/vulkan/core.py:4696-4760):
    the same meshes with the same topology, and new vertex positions only
    for meshes marked ``deformable``."""
    if (len(old.mesh_sources) != len(new.mesh_sources)
            or any(a is not b for a, b in zip(old.mesh_sources, new.mesh_sources))
            or not np.array_equal(old.mesh_vertex_offset, new.mesh_vertex_offset)
            or not np.array_equal(old.mesh_triangle_offset, new.mesh_triangle_offset)
            or not np.array_equal(old.instance_mesh, new.instance_mesh)
            or old.environment_kind != new.environment_kind
            or (old.environment_image is None) != (new.environment_image is None)
            or (old.environment_image is not None and old.environment_image.shape != new.environment_image.shape)
            or (old.volume is None) != (new.volume is None)):
        return None
    if old.volume is not None and np.shape(old.volume["density"]) != np.shape(new.volume["density"]):
        return None
    mask = np.zeros(len(new.mesh_sources), np.uint8)
    for m, source in enumerate(new.mesh_sources):
        v0, v1 = int(new.mesh_vertex_offset[m]), int(new.mesh_vertex_offset[m + 1])
        t0, t1 = int(new.mesh_triangle_offset[m]), int(new.mesh_triangle_offset[m + 1])
        if not np.array_equal(old.indices[t0:t1], new.indices[t0:t1]):
            return None
        moved = not np.array_equal(old.vertices[v0:v1], new.vertices[v0:v1])
        if moved and not getattr(source, "deformable", False):
            return None
        if moved or not np.array_equal(old.normals[v0:v1], new.normals[v0:v1]):
            mask[m] = 1
    return mask


def camera_kind(camera) -> int:
    name = type(camera).__name__
    if name == "PanoramicCamera" or hasattr(camera, "horizontal_fov_degrees"):
        return _native.PROJECTION_PANORAMIC
    if name == "OrthographicCamera" or hasattr(camera, "vertical_size"):
        return _native.PROJECTION_ORTHOGRAPHIC
    return _native.PROJECTION_PERSPECTIVE


def camera_basis(camera):
    """Camera frame in float32, computed as ReferencePathTracer._camera_rays
    does (path_tracer.py:110-116)."""
    position = np.asarray(camera.position, dtype=np.float32)
    forward = np.asarray(camera.target, dtype=np.float32) - position
    forward /= np.linalg.norm(forward)
    right = np.cross(forward, np.asarray(camera.up, dtype=np.float32))
    right /= np.linalg.norm(right)
    up = np.cross(right, forward)
    return position, forward, right, up


def pack_camera(camera) -> _native.OlcCamera:
    position, forward, right, up = camera_basis(camera)
    cam = _native.OlcCamera()
    for k in range(3):
        cam.position[k] = float(position[k])
        cam.forward[k] = float(forward[k])
        cam.right[k] = float(right[k])
        cam.up[k] = float(up[k])
    kind = camera_kind(camera)
    cam.projection = kind
    if kind == _native.PROJECTION_PANORAMIC:
        cam.horizontal_half = math.radians(camera.horizontal_fov_degrees) * 0.5
        cam.vertical_half = math.radians(camera.vertical_fov_degrees) * 0.5
    elif kind == _native.PROJECTION_ORTHOGRAPHIC:
        cam.half_height = float(camera.vertical_size) * 0.5
    else:
        cam.half_height = math.tan(math.radians(camera.vertical_fov_degrees) / 2.0)
    return cam
