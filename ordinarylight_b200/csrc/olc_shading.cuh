// Shading math: environment/sky, the GGX + Lambert BSDF, emitter sampling.
//
// Production BSDF = the reference's isotropic PBR helpers
// (ordinarylight_pbr_cosine_hemisphere / _evaluate / _pdf /
// _sample_half_vector / _reflect / _weight / _specular_probability,
// ordinarylight/shaders/ordinaryshade_primary.glsl:506-609):
//   f0 = mix(0.04, base, metallic); F = Schlick(f0, v.h);
//   D = GGX with alpha = max(roughness^2, 0.0009) (not capped, see ggx_d);
//   G = Smith G1(n.v) G1(n.l);
//   f = (1 - F)(1 - metallic) base / pi + F D G / (4 n.v n.l);
//   specular lobe probability = clamp(max(f0), 0.1, 0.9);
//   pdf = mix(n.l / pi, D n.h / (4 v.h), p_spec).
// Reference-compatible BSDF = the CPU tracer's Lambert: throughput *= albedo,
// cosine-distributed direction (path_tracer.py:84-87, :205-211).
#pragma once

#include "olc_common.cuh"

#define OLC_PI 3.14159265358979f

// CPU reference sky (path_tracer.py:201-202).
OLC_D float3 cpu_sky(float3 d) {
  float blend = clampf(0.5f * (d.y + 1.0f), 0.0f, 1.0f);
  return f3(0.8f, 0.8f, 0.8f) * (1.0f - blend) + f3(0.2f, 0.4f, 0.9f) * blend;
}

// Reference GPU analytic sky (ordinaryshade_primary.glsl:703-707).
OLC_D float3 gpu_sky(float3 d) {
  float sky = fmaxf(d.y, 0.0f);
  return lerp3(f3(0.018f, 0.022f, 0.032f), f3(0.32f, 0.46f, 0.72f), sky);
}

// Environment radiance (constant or equirectangular nearest lookup as in
// ReferencePathTracer._sky, path_tracer.py:185-200); kind NONE falls back to
// the mode's analytic sky.
OLC_D float3 environment_radiance(const SceneRec& s, float3 d, bool cpu_mode) {
  if (s.env_kind == 0u) return cpu_mode ? cpu_sky(d) : gpu_sky(d);
  if (s.env_kind == 1u) return f3(s.env_color);
  float lon = atan2f(d.z, d.x) + s.env_rotation;
  float u = lon / (2.0f * OLC_PI) + 0.5f;
  u = u - floorf(u);
  float v = acosf(clampf(d.y, -1.0f, 1.0f)) / OLC_PI;
  uint32_t x = min((uint32_t)(u * (float)s.env_w), s.env_w - 1u);
  uint32_t y = min((uint32_t)(v * (float)s.env_h), s.env_h - 1u);
  const float* p = s.env_image + 3ull * ((uint64_t)y * s.env_w + x);
  return f3(p[0], p[1], p[2]) * f3(s.env_color);
}

OLC_D void tangent_frame(float3 n, float3& t, float3& b) {
  t = (fabsf(n.z) < 0.999f) ? cross(n, f3(0.0f, 0.0f, 1.0f)) : cross(n, f3(0.0f, 1.0f, 0.0f));
  t = normalize(t);
  b = cross(n, t);
}

OLC_D float3 cosine_hemisphere(float3 n, float u, float v) {
  float r = sqrtf(u);
  float phi = 2.0f * OLC_PI * v;
  float3 t, b;
  tangent_frame(n, t, b);
  float sp, cp;
  __sincosf(phi, &sp, &cp);
  return normalize(t * (r * cp) + b * (r * sp) + n * sqrtf(fmaxf(0.0f, 1.0f - u)));
}

// The CPU reference's bounce direction: normalize(n + s) with s uniform on
// the unit sphere and flipped into n's hemisphere
// (ReferencePathTracer._cosine_hemisphere, path_tracer.py:205-211).  The flip
// makes this distribution more concentrated around n than a cosine lobe
// (normalize(n + s) is cosine-distributed only for s on the whole sphere),
// while the reference still weights the bounce by the albedo alone;
// reference-compatible mode reproduces the reference's estimator exactly in
// distribution, so it uses the same construction.
OLC_D float3 reference_bounce_direction(float3 n, float u, float v) {
  float z = 1.0f - 2.0f * u;
  float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  float sp, cp;
  __sincosf(2.0f * OLC_PI * v, &sp, &cp);
  float3 s = f3(r * cp, r * sp, z);
  if (dot(s, n) < 0.0f) s = -s;
  return normalize(n + s);
}

OLC_D float ggx_alpha2(float roughness) {
  float a = fmaxf(roughness * roughness, 0.0009f);
  return a * a;
}
// GGX distribution a2 / (pi ((n.h)^2 (a2 - 1) + 1)^2), with the bracket
// written as |n x h|^2 + (n.h)^2 a2 (the same value for unit vectors) so that
// float32 resolves it near the peak, where 1 + (n.h)^2 (a2 - 1) cancels.  The
// reference floors pi den^2 at 1e-6, which caps D near the peak for
// roughness below about 0.155 while its sampler still draws the uncapped
// distribution: f cos / pdf then no longer integrates f, and estimators of
// one scene disagree (by a fifth at roughness 0.05).  Here D is the GGX
// distribution the sampler draws; above roughness 0.155 the two are equal.
OLC_D float ggx_d(float nh, float s2, float a2) {
  float den = s2 + nh * nh * a2;
  return a2 / fmaxf(OLC_PI * den * den, 1e-30f);
}
// |n x h|^2 for the GGX bracket (1 where n.h <= 0, whose terms vanish).
OLC_D float sin2_between(float3 n, float3 h, float nh) {
  if (!(nh > 0.0f)) return 1.0f;
  const float3 c = cross(n, h);
  return dot(c, c);
}
OLC_D float ggx_g1(float nd, float a2) {
  return 2.0f * nd / fmaxf(nd + sqrtf(a2 + (1.0f - a2) * nd * nd), 1e-6f);
}

struct SurfaceMat {
  float3 base;
  float roughness;
  float3 emission;
  float metallic;
  uint32_t two_sided;
  float transmission;
  float ior;
};

OLC_D float spec_probability(const SurfaceMat& m) {
  float3 f0 = lerp3(f3(0.04f, 0.04f, 0.04f), m.base, m.metallic);
  return clampf(max3(f0), 0.1f, 0.9f);
}

OLC_D float3 pbr_eval(const SurfaceMat& m, float3 n, float3 view, float3 out) {
  float nv = fmaxf(dot(n, view), 0.0f);
  float nl = fmaxf(dot(n, out), 0.0f);
  if (nv <= 0.0f || nl <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
  float3 h = normalize(view + out);
  float nh = fmaxf(dot(n, h), 0.0f);
  float vh = fmaxf(dot(view, h), 0.0f);
  float3 f0 = lerp3(f3(0.04f, 0.04f, 0.04f), m.base, m.metallic);
  float w = 1.0f - clampf(vh, 0.0f, 1.0f);
  float w5 = w * w * w * w * w;
  float3 F = f0 + (f3(1.0f, 1.0f, 1.0f) - f0) * w5;
  float a2 = ggx_alpha2(m.roughness);
  float D = ggx_d(nh, sin2_between(n, h, nh), a2);
  float G = ggx_g1(nv, a2) * ggx_g1(nl, a2);
  float3 spec = F * (D * G / fmaxf(4.0f * nv * nl, 1e-6f));
  float3 diff = (f3(1.0f, 1.0f, 1.0f) - F) * m.base * ((1.0f - m.metallic) / OLC_PI);
  return diff + spec;
}

OLC_D float pbr_pdf(const SurfaceMat& m, float3 n, float3 view, float3 out) {
  float nl = fmaxf(dot(n, out), 0.0f);
  if (nl <= 0.0f) return 0.0f;
  float3 h = normalize(view + out);
  float nh = fmaxf(dot(n, h), 0.0f);
  float vh = fmaxf(dot(view, h), 1e-6f);
  float a2 = ggx_alpha2(m.roughness);
  float spec_pdf = ggx_d(nh, sin2_between(n, h, nh), a2) * nh / (4.0f * vh);
  float diff_pdf = nl / OLC_PI;
  float p = spec_probability(m);
  return diff_pdf + (spec_pdf - diff_pdf) * p;
}

OLC_D float3 sample_half_vector(float3 n, float roughness, float u, float v) {
  float a2 = ggx_alpha2(roughness);
  float phi = 2.0f * OLC_PI * v;
  // cos^2 = (1 - u) / (1 + (a2 - 1) u) and sin^2 = a2 u / (1 + (a2 - 1) u),
  // the bracket as (1 - u) + a2 u and sin from its own ratio: both forms
  // with 1 - ... cancel in float32 for narrow lobes
  const float den = fmaxf(fmaf(a2, u, 1.0f - u), 1e-30f);
  float c = sqrtf((1.0f - u) / den);
  float sn = sqrtf(a2 * u / den);
  float3 t, b;
  tangent_frame(n, t, b);
  float sp, cp;
  __sincosf(phi, &sp, &cp);
  return normalize(t * (sn * cp) + b * (sn * sp) + n * c);
}

// BSDF sampling after samplePbr (transport_v1/lighting.glsl:226-246): lobe
// choice with the specular probability, a cosine-weighted diffuse direction
// or a GGX half-vector reflection, pdf = mix(diffuse pdf, specular pdf, p)
// and weight = f cos / pdf.  One deliberate difference: the reference
// replaces a specular reflection that points below the surface with a fresh
// cosine direction but still reports the mixture pdf, which under-states the
// density of the directions it returns (the estimator comes out too bright,
// most visibly for rough surfaces).  Here such a sample is invalid — zero
// weight, the path ends — so the reported pdf is exactly the density of the
// directions that carry weight and the estimator is unbiased.  Returns false
// for an invalid sample.
OLC_D bool pbr_sample(const SurfaceMat& m, float3 n, float3 incoming, uint32_t& rng, float3& out, float3& weight,
                      float& pdf) {
  float3 view = -incoming;
  float p = spec_probability(m);
  bool specular = olc_rand(rng) < p;
  float u = olc_rand(rng), v = olc_rand(rng);
  if (specular) {
    float3 h = sample_half_vector(n, m.roughness, u, v);
    out = incoming - h * (2.0f * dot(h, incoming));
  } else {
    out = cosine_hemisphere(n, u, v);
  }
  out = normalize(out);
  if (!(dot(n, out) > 0.0f)) {
    weight = f3(0.0f, 0.0f, 0.0f);
    pdf = 0.0f;
    return false;
  }
  pdf = fmaxf(pbr_pdf(m, n, view, out), 1e-6f);
  float3 f = pbr_eval(m, n, view, out);
  weight = f * (fmaxf(dot(n, out), 0.0f) / pdf);
  return true;
}

OLC_D float power_heuristic(float a, float b) {
  float a2 = a * a, b2 = b * b;
  return a2 / fmaxf(a2 + b2, 1e-6f);
}

OLC_D SurfaceMat load_material(const SceneView& s, uint32_t mi) {
  MaterialRec r = s.materials[mi];
  SurfaceMat m;
  m.base = f3(r.base_rough);
  m.roughness = r.base_rough.w;
  m.emission = f3(r.emit_metal);
  m.metallic = r.emit_metal.w;
  const MaterialAux aux = s.material_aux[mi];
  m.two_sided = aux.two_sided;
  m.transmission = aux.transmission;
  m.ior = aux.ior;
  return m;
}

// Emitter selection with the probabilities of the power CDF
// (sampleAreaLightTechnique, transport_v1/lighting.glsl:356-377) through an
// alias table: one 8-byte load instead of a dependent binary search.
// Returns the global emitter index (scene base + scene-local index).
OLC_D uint32_t select_emitter(const SceneView& s, const SceneRec& sc, float u) {
  float scaled = u * (float)sc.num_emitters;
  uint32_t i = min((uint32_t)scaled, sc.num_emitters - 1u);
  float frac = scaled - (float)i;
  AliasEntry e = s.emitter_alias[sc.emitter_base + i];
  return sc.emitter_base + (frac < e.threshold ? i : e.alias);
}

OLC_D EmitterRec load_emitter(const SceneView& s, uint32_t i) {
  const float4* p = reinterpret_cast<const float4*>(s.emitters + i);
  EmitterRec e;
  e.a_pdf = __ldg(p + 0);
  e.e1_area = __ldg(p + 1);
  e.e2_sided = __ldg(p + 2);
  e.normal = __ldg(p + 3);
  e.emission = __ldg(p + 4);
  return e;
}

// Point of barycentrics (b1, b2) on the emitter: a + b1 (b - a) + b2 (c - a).
// Uniform area sampling uses b1 = sqrt(u)(1 - v), b2 = sqrt(u) v, the
// mapping of ordinarylight_area_light_position (ordinaryshade_primary.glsl:668-671).
// The fused multiply-adds are written out so that every kernel (ReSTIR's
// light pool, its reuse passes, shading) computes the same point bit for bit.
OLC_D float3 emitter_point(const EmitterRec& e, float b1, float b2) {
  return f3(__fmaf_rn(e.e2_sided.x, b2, __fmaf_rn(e.e1_area.x, b1, e.a_pdf.x)),
            __fmaf_rn(e.e2_sided.y, b2, __fmaf_rn(e.e1_area.y, b1, e.a_pdf.y)),
            __fmaf_rn(e.e2_sided.z, b2, __fmaf_rn(e.e1_area.z, b1, e.a_pdf.z)));
}

OLC_D float emitter_cosine(const EmitterRec& e, float3 dir) {
  float c = -dot(f3(e.normal), dir);
  return e.e2_sided.w > 0.5f ? fabsf(c) : fmaxf(c, 0.0f);
}
