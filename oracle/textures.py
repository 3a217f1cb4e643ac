"""ORACLE — test infrastructure only, never part of the product path.

numpy restatement of the reference's material texture lookups
(ordinarylight/shaders/wavefront_textures.glsl) on the packed texture words
of Scene.texture_data and the bindings of Scene.texture_binding_data, in
float32 like the shader:

* wrapTextureCoordinate / wrapTextureIndex (:22-53): repeat, clamp, mirror;
* decodeTextureTexel (:55-66): unorm8, sRGB through the 256-entry table;
* sampleTextureLevel (:91-109): nearest or bilinear at texel centres;
* sampleMaterialTexture (:134-204): KHR transform (offset + rotation of the
  scaled UV), LOD = clamp(log2(max(footprint * scale * max(w, h), 1)), 0,
  levels - 1), trilinear between LOD floor and floor + 1 when linear;
* ordinarylight_texture_apply_normal (ordinaryshade_primary.glsl:367-381).
"""

from __future__ import annotations

import numpy as np

F = np.float32


def srgb_table():
    c = np.arange(256, dtype=np.float64) / 255.0
    return np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4).astype(F)


def _wrap_coordinate(v, mode):
    v = v.astype(F)
    if mode == 1:
        return np.clip(v, F(0.0), F(0.99999994))
    if mode == 2:
        period = (v - F(2.0) * np.floor(v * F(0.5))).astype(F)
        period = np.where(period < 0, period + F(2.0), period)
        return np.where(period <= 1.0, period, F(2.0) - period).astype(F)
    return (v - np.floor(v)).astype(F)


def _wrap_index(v, size, mode):
    if mode == 1:
        return np.clip(v, 0, size - 1)
    period = size * 2 if mode == 2 else size
    w = np.fmod(v, period)
    w = np.where(w < 0, w + period, w)
    if mode == 2:
        w = np.where(w >= size, (period - 1) - w, w)
    return w


def _decode(words, srgb, lut):
    r = (words & 255).astype(np.int64)
    g = ((words >> 8) & 255).astype(np.int64)
    b = ((words >> 16) & 255).astype(np.int64)
    a = (words >> 24).astype(np.int64)
    if srgb:
        rgb = [lut[r], lut[g], lut[b]]
    else:
        rgb = [r.astype(F) / F(255.0), g.astype(F) / F(255.0), b.astype(F) / F(255.0)]
    return np.stack(rgb + [a.astype(F) / F(255.0)], axis=-1).astype(F)


def _mix(a, b, t):
    t = t[..., None].astype(F)
    return (a * (F(1.0) - t) + b * t).astype(F)


def sample_level(words, base_offset, bw, bh, level, u, v, wrap_s, wrap_t, srgb, linear, lut):
    sx = max((bw + (1 << level) - 1) >> level, 1)
    sy = max((bh + (1 << level) - 1) >> level, 1)
    offset, w, h = base_offset, bw, bh
    for _ in range(level):
        offset += w * h
        w, h = max((w + 1) // 2, 1), max((h + 1) // 2, 1)
    wu, wv = _wrap_coordinate(u, wrap_s), _wrap_coordinate(v, wrap_t)

    def fetch(cx, cy):
        x = _wrap_index(cx, sx, wrap_s)
        y = _wrap_index(cy, sy, wrap_t)
        return _decode(words[offset + y * sx + x], srgb, lut)

    if not linear:
        return fetch(np.floor(wu * F(sx)).astype(np.int64), np.floor(wv * F(sy)).astype(np.int64))
    tx = (wu * F(sx) - F(0.5)).astype(F)
    ty = (wv * F(sy) - F(0.5)).astype(F)
    x0, y0 = np.floor(tx).astype(np.int64), np.floor(ty).astype(np.int64)
    fx, fy = (tx - np.floor(tx)).astype(F), (ty - np.floor(ty)).astype(F)
    top = _mix(fetch(x0, y0), fetch(x0 + 1, y0), fx)
    bottom = _mix(fetch(x0, y0 + 1), fetch(x0 + 1, y0 + 1), fx)
    return _mix(top, bottom, fy)


def sample_material_texture(words, bindings, binding, uv0, uv1, srgb, fp0, fp1, lut=None):
    """words: uint32 texture words; bindings: (n, 8) float32 records."""
    lut = srgb_table() if lut is None else lut
    n = len(uv0)
    if binding < 0:
        return np.ones((n, 4), F)
    rec = np.asarray(bindings[binding], F)
    texture = int(rec[0])
    if texture < 0 or texture >= int(words[0]):
        return np.ones((n, 4), F)
    use_uv1 = rec[3] > 0.5
    uv = np.asarray(uv1 if use_uv1 else uv0, F)
    fp = np.asarray(fp1 if use_uv1 else fp0, F)
    cs, sn = rec[1], rec[2]
    su, sv = uv[:, 0] * rec[6], uv[:, 1] * rec[7]
    u = (rec[4] + (cs * su - sn * sv)).astype(F)
    v = (rec[5] + (sn * su + cs * sv)).astype(F)
    fp = (fp * max(abs(rec[6]), abs(rec[7]))).astype(F)
    meta = words[1 + 8 * texture: 9 + 8 * texture]
    offset = int(meta[0] if srgb else meta[1])
    w, h, flags, levels = int(meta[2]), int(meta[3]), int(meta[4]), int(meta[5])
    wrap_s, wrap_t, linear = flags & 3, (flags >> 2) & 3, (flags & 16) != 0
    lod = np.clip(np.log2(np.maximum(fp * F(max(w, h)), F(1.0))).astype(F), F(0.0), F(max(levels, 1) - 1))
    lower = np.floor(lod).astype(np.int64)
    out = np.empty((n, 4), F)
    for level in np.unique(lower):
        sel = lower == level
        first = sample_level(words, offset, w, h, int(level), u[sel], v[sel], wrap_s, wrap_t, srgb, linear, lut)
        if linear and level + 1 < levels:
            second = sample_level(words, offset, w, h, int(level) + 1, u[sel], v[sel], wrap_s, wrap_t, srgb, True,
                                  lut)
            first = _mix(first, second, (lod[sel] - np.floor(lod[sel])).astype(F))
        out[sel] = first
    return out


def apply_normal(sampled, normal_scale, n, tangent_data, cs, sn, scale_u, scale_v):
    def norm(x):
        return x / np.linalg.norm(x, axis=-1, keepdims=True)

    tn = sampled[:, :3] * 2.0 - 1.0
    tn[:, :2] *= normal_scale
    tn = norm(tn)
    td = tangent_data[:, :3]
    t = norm(td - n * np.sum(n * td, axis=1, keepdims=True))
    b = np.cross(n, t) * tangent_data[:, 3:4]
    tt = norm(t * (cs / scale_u) + b * (-sn / scale_v))
    tb = norm(t * (sn / scale_u) + b * (cs / scale_v))
    return norm(tt * tn[:, :1] + tb * tn[:, 1:2] + n * tn[:, 2:3])
