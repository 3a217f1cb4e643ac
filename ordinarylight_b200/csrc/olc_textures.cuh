// Material textures: sampling of the packed RGBA8 mip pyramids and their
// application to a surface's material and shading normal.  Restates the
// reference's generated texture helpers in CUDA:
//   wrap / fetch / bilinear level sample   wavefront_textures.glsl:22-109
//   material texture sample (KHR transform, ray-cone LOD, trilinear)
//                                          wavefront_textures.glsl:134-204
//   applyMaterialTextures                  wavefront_textures.glsl:207-272
//   normal map (ordinarylight_texture_apply_normal)
//                                          ordinaryshade_primary.glsl:367-381
//   triangle tangent and UV density        wavefront_textures.glsl:190-197,
//                                          ordinaryshade_primary.glsl:321-345
// The packing (texture words, bindings, per-material binding records) is
// the reference's Scene.texture_data / texture_binding_data layout.
#pragma once

#include "olc_common.cuh"
#include "olc_shading.cuh"

namespace olc {

OLC_D float tex_fract(float v) { return v - floorf(v); }

// wrapTextureCoordinate: 0 repeat, 1 clamp, 2 mirror.
OLC_D float wrap_coordinate(float value, uint32_t mode) {
  if (mode == 1u) return clampf(value, 0.0f, 0.99999994f);
  if (mode == 2u) {
    float period = value - 2.0f * floorf(value * 0.5f);   // GLSL mod(value, 2)
    if (period < 0.0f) period += 2.0f;
    return period <= 1.0f ? period : 2.0f - period;
  }
  return tex_fract(value);
}

OLC_D int wrap_index(int value, int size, uint32_t mode) {
  if (mode == 1u) return min(max(value, 0), size - 1);
  const int period = mode == 2u ? size * 2 : size;
  int wrapped = value % period;
  if (wrapped < 0) wrapped += period;
  return (mode == 2u && wrapped >= size) ? (period - 1) - wrapped : wrapped;
}

OLC_D float4 decode_texel(uint32_t packed, bool srgb, const float* lut) {
  const float r = (float)(packed & 255u), g = (float)((packed >> 8) & 255u), b = (float)((packed >> 16) & 255u),
              a = (float)(packed >> 24);
  if (!srgb) return make_float4(r / 255.0f, g / 255.0f, b / 255.0f, a / 255.0f);
  return make_float4(lut[packed & 255u], lut[(packed >> 8) & 255u], lut[(packed >> 16) & 255u], a / 255.0f);
}

OLC_D float4 fetch_texel(const uint32_t* words, uint32_t offset, int sx, int sy, int cx, int cy, uint32_t wrap_s,
                         uint32_t wrap_t, bool srgb, const float* lut) {
  const int x = wrap_index(cx, sx, wrap_s), y = wrap_index(cy, sy, wrap_t);
  return decode_texel(__ldg(words + offset + (uint32_t)(y * sx + x)), srgb, lut);
}

OLC_D float4 mix4(float4 a, float4 b, float t) {
  return make_float4(a.x * (1.0f - t) + b.x * t, a.y * (1.0f - t) + b.y * t, a.z * (1.0f - t) + b.z * t,
                     a.w * (1.0f - t) + b.w * t);
}

// sampleTextureLevel: nearest or bilinear lookup of mip `level`.
OLC_D float4 sample_level(const uint32_t* words, uint32_t base_offset, int bw, int bh, uint32_t level, float u,
                          float v, uint32_t wrap_s, uint32_t wrap_t, bool srgb, bool linear, const float* lut) {
  const int sx = max((bw + (1 << level) - 1) >> level, 1), sy = max((bh + (1 << level) - 1) >> level, 1);
  uint32_t offset = base_offset;
  int w = bw, h = bh;
  for (uint32_t l = 0; l < level; ++l) {
    offset += (uint32_t)(w * h);
    w = max((w + 1) / 2, 1);
    h = max((h + 1) / 2, 1);
  }
  const float wu = wrap_coordinate(u, wrap_s), wv = wrap_coordinate(v, wrap_t);
  if (!linear)
    return fetch_texel(words, offset, sx, sy, (int)floorf(wu * (float)sx), (int)floorf(wv * (float)sy), wrap_s, wrap_t,
                       srgb, lut);
  const float tx = wu * (float)sx - 0.5f, ty = wv * (float)sy - 0.5f;
  const int x0 = (int)floorf(tx), y0 = (int)floorf(ty);
  const float fx = tex_fract(tx), fy = tex_fract(ty);
  const float4 top = mix4(fetch_texel(words, offset, sx, sy, x0, y0, wrap_s, wrap_t, srgb, lut),
                          fetch_texel(words, offset, sx, sy, x0 + 1, y0, wrap_s, wrap_t, srgb, lut), fx);
  const float4 bottom = mix4(fetch_texel(words, offset, sx, sy, x0, y0 + 1, wrap_s, wrap_t, srgb, lut),
                             fetch_texel(words, offset, sx, sy, x0 + 1, y0 + 1, wrap_s, wrap_t, srgb, lut), fx);
  return mix4(top, bottom, fy);
}

// sampleMaterialTexture: binding < 0 (or a missing texture) reads as white.
OLC_D float4 sample_material_texture(const SceneRec& sc, float binding_value, float2 uv0, float2 uv1, bool srgb,
                                     float footprint0, float footprint1) {
  const int binding = (int)binding_value;
  if (binding < 0) return make_float4(1.0f, 1.0f, 1.0f, 1.0f);
  const float4 tr = sc.tex_bindings[2 * binding], os = sc.tex_bindings[2 * binding + 1];
  const int texture = (int)tr.x;
  const uint32_t* words = sc.tex_words;
  if (texture < 0 || (uint32_t)texture >= words[0]) return make_float4(1.0f, 1.0f, 1.0f, 1.0f);
  const bool use_uv1 = tr.w > 0.5f;
  float2 uv = use_uv1 ? uv1 : uv0;
  float footprint = use_uv1 ? footprint1 : footprint0;
  const float cs = tr.y, sn = tr.z;
  const float su = uv.x * os.z, sv = uv.y * os.w;
  uv = make_float2(os.x + (cs * su - sn * sv), os.y + (sn * su + cs * sv));
  footprint = footprint * fmaxf(fabsf(os.z), fabsf(os.w));
  const uint32_t* meta = words + 1u + 8u * (uint32_t)texture;
  const uint32_t offset = meta[srgb ? 0 : 1];
  const int w = (int)meta[2], h = (int)meta[3];
  const uint32_t flags = meta[4], levels = meta[5];
  const uint32_t wrap_s = flags & 3u, wrap_t = (flags >> 2) & 3u;
  const float lod =
      clampf(log2f(fmaxf(footprint * (float)max(w, h), 1.0f)), 0.0f, (float)(max(levels, 1u) - 1u));
  const uint32_t lower = (uint32_t)floorf(lod);
  const bool linear = (flags & 16u) != 0u;
  const float4 first = sample_level(words, offset, w, h, lower, uv.x, uv.y, wrap_s, wrap_t, srgb, linear, sc.srgb_lut);
  if (!linear || lower + 1u >= levels) return first;
  const float4 second =
      sample_level(words, offset, w, h, lower + 1u, uv.x, uv.y, wrap_s, wrap_t, srgb, true, sc.srgb_lut);
  return mix4(first, second, tex_fract(lod));
}

// sqrt(UV area / world area) of a triangle: texels per world unit for the
// ray-cone footprint.
OLC_D float triangle_uv_density(float3 a, float3 b, float3 c, float2 ua, float2 ub, float2 uc) {
  const float2 e0 = make_float2(ub.x - ua.x, ub.y - ua.y), e1 = make_float2(uc.x - ua.x, uc.y - ua.y);
  const float uv_area = fabsf(e0.x * e1.y - e0.y * e1.x);
  const float world_area = length(cross(b - a, c - a));
  return sqrtf(uv_area / fmaxf(world_area, 1e-8f));
}

// Tangent (xyz) and handedness (w) of a triangle from its UV gradients.
OLC_D float4 triangle_tangent(float3 a, float3 b, float3 c, float2 ua, float2 ub, float2 uc, float3 n) {
  const float3 ea = b - a, eb = c - a;
  const float2 da = make_float2(ub.x - ua.x, ub.y - ua.y), db = make_float2(uc.x - ua.x, uc.y - ua.y);
  const float det = da.x * db.y - da.y * db.x;
  if (fabsf(det) < 1e-8f) {
    const float3 fallback = fabsf(n.z) < 0.999f ? cross(n, f3(0.0f, 0.0f, 1.0f)) : cross(n, f3(0.0f, 1.0f, 0.0f));
    const float3 t = normalize(fallback);
    return make_float4(t.x, t.y, t.z, 1.0f);
  }
  const float inv = 1.0f / det;
  const float3 t = normalize((ea * db.y - eb * da.y) * inv);
  const float3 bt = normalize((eb * da.x - ea * db.x) * inv);
  const float hand = dot(cross(n, t), bt) < 0.0f ? -1.0f : 1.0f;
  return make_float4(t.x, t.y, t.z, hand);
}

// Tangent-space normal map sample -> world shading normal.
OLC_D float3 apply_normal_map(float3 sampled, float normal_scale, float3 n, float4 tangent_data, float cs, float sn,
                              float scale_u, float scale_v) {
  float3 tn = sampled * 2.0f - f3(1.0f, 1.0f, 1.0f);
  tn.x *= normal_scale;
  tn.y *= normal_scale;
  tn = normalize(tn);
  const float3 td = f3(tangent_data.x, tangent_data.y, tangent_data.z);
  const float3 t = normalize(td - n * dot(n, td));
  const float3 b = cross(n, t) * tangent_data.w;
  const float iu = 1.0f / scale_u, iv = 1.0f / scale_v;
  const float3 tt = normalize(t * (cs * iu) + b * (-sn * iv));
  const float3 tb = normalize(t * (sn * iu) + b * (cs * iv));
  return normalize(tt * tn.x + tb * tn.y + n * tn.z);
}

// Per-vertex attributes of triangle slot `slot` (uv0.xy uv1.xy, then
// object-space tangent xyz + handedness, for each of the 3 vertices).
OLC_D void load_slot_attributes(const SceneRec& sc, uint32_t slot, float4 uv[3], float4 tan[3]) {
  const float4* a = sc.tex_attr + 6ull * (slot - sc.slot_base);
  for (int k = 0; k < 3; ++k) {
    uv[k] = a[2 * k];
    tan[k] = a[2 * k + 1];
  }
}

struct TexturedHit {
  SurfaceMat m;
  float3 ns;
  float occlusion;
};

// Apply the material's textures at a hit (applyMaterialTextures and the
// normal map of wavefront_shade.comp:368-391): the material's base colour,
// emission, transmission, roughness and metallic and the shading normal
// (oriented towards ng) change, and the occlusion factor of the BSDF sample
// weight is returned with them.  v0..v2: world vertices; tri_normals: the
// slot's object-space vertex normals; ns: the interpolated world shading
// normal; cone_width: the ray cone's width at the hit (0 for camera rays).
// Out of line: the textured path's registers do not burden its callers.
static __device__ __noinline__ TexturedHit apply_textures(const SceneRec& sc, uint32_t material_local, uint32_t slot,
                                                          float3 v0, float3 v1, float3 v2, Affine o2w, Affine w2o,
                                                          const float4* tri_normals, float bu, float bv,
                                                          float cone_width, float3 ng, float3 ns, SurfaceMat m) {
  const float4 i0 = sc.mat_tex[3 * material_local], i1 = sc.mat_tex[3 * material_local + 1],
               i2 = sc.mat_tex[3 * material_local + 2];
  if (i0.x < 0.0f && i0.y < 0.0f && i0.z < 0.0f && i0.w < 0.0f && i1.x < 0.0f && i1.y < 0.0f)
    return TexturedHit{m, ns, 1.0f};
  float4 uv[3], tan[3];
  load_slot_attributes(sc, slot, uv, tan);
  const float w0 = (1.0f - bu) - bv;
  const float2 uv0 = make_float2(uv[0].x * w0 + uv[1].x * bu + uv[2].x * bv, uv[0].y * w0 + uv[1].y * bu + uv[2].y * bv);
  float2 uv1 = make_float2(0.0f, 0.0f);
  const float density0 = triangle_uv_density(v0, v1, v2, make_float2(uv[0].x, uv[0].y), make_float2(uv[1].x, uv[1].y),
                                             make_float2(uv[2].x, uv[2].y));
  const float fp0 = cone_width * density0;
  float fp1 = 0.0f;
  if (i2.x > 0.5f) {
    uv1 = make_float2(uv[0].z * w0 + uv[1].z * bu + uv[2].z * bv, uv[0].w * w0 + uv[1].w * bu + uv[2].w * bv);
    fp1 = cone_width * triangle_uv_density(v0, v1, v2, make_float2(uv[0].z, uv[0].w), make_float2(uv[1].z, uv[1].w),
                                           make_float2(uv[2].z, uv[2].w));
  }
  m.transmission *= sample_material_texture(sc, i1.y, uv0, uv1, false, fp0, fp1).x;
  const float4 base = sample_material_texture(sc, i0.x, uv0, uv1, true, fp0, fp1);
  m.base = m.base * f3(base.x, base.y, base.z);
  const float4 emit = sample_material_texture(sc, i0.z, uv0, uv1, true, fp0, fp1);
  m.emission = m.emission * f3(emit.x, emit.y, emit.z);
  float occlusion = 1.0f;
  if (!(m.transmission > 0.001f)) {
    const float4 mr = sample_material_texture(sc, i0.y, uv0, uv1, false, fp0, fp1);
    m.roughness *= mr.y;
    m.metallic *= mr.z;
    const float occ = sample_material_texture(sc, i1.x, uv0, uv1, false, fp0, fp1).x;
    occlusion = 1.0f * (1.0f - i1.w) + occ * i1.w;   // mix(1, occlusion, strength)
  }
  const int normal_binding = (int)i0.w;
  if (normal_binding >= 0) {
    const float4 nb_tr = sc.tex_bindings[2 * normal_binding], nb_os = sc.tex_bindings[2 * normal_binding + 1];
    float4 tangent_data;
    if (nb_tr.w > 0.5f) {
      tangent_data = triangle_tangent(v0, v1, v2, make_float2(uv[0].z, uv[0].w), make_float2(uv[1].z, uv[1].w),
                                      make_float2(uv[2].z, uv[2].w), ns);
    } else {
      // world tangents per vertex, orthogonalised against the vertex's world
      // normal (Mesh.world_tangents, scene/_core.py:702-714), interpolated
      const float det = o2w.r0.x * (o2w.r1.y * o2w.r2.z - o2w.r1.z * o2w.r2.y) -
                        o2w.r0.y * (o2w.r1.x * o2w.r2.z - o2w.r1.z * o2w.r2.x) +
                        o2w.r0.z * (o2w.r1.x * o2w.r2.y - o2w.r1.y * o2w.r2.x);
      const float weights[3] = {w0, bu, bv};
      float4 acc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      for (int k = 0; k < 3; ++k) {
        float3 t = xform_vector(o2w, f3(tan[k].x, tan[k].y, tan[k].z));
        const float3 nw = normalize(xform_normal_by_inverse(w2o, f3(tri_normals[k])));
        t = normalize(t - nw * dot(t, nw));
        const float hand = det < 0.0f ? -tan[k].w : tan[k].w;
        acc.x += t.x * weights[k];
        acc.y += t.y * weights[k];
        acc.z += t.z * weights[k];
        acc.w += hand * weights[k];
      }
      tangent_data = acc;
    }
    const float4 s = sample_material_texture(sc, i0.w, uv0, uv1, false, fp0, fp1);
    ns = apply_normal_map(f3(s.x, s.y, s.z), i1.z, ns, tangent_data, nb_tr.y, nb_tr.z, nb_os.z, nb_os.w);
    if (dot(ns, ng) < 0.0f) ns = -ns;
  }
  return TexturedHit{m, ns, occlusion};
}

}  // namespace olc
