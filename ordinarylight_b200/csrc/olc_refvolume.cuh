// The reference CPU renderer's volume model, for the reference-compatible
// mode: every ray segment of a path crosses the scene's visible volumes
// before its hit or miss is shaded (ReferencePathTracer.render_hdr,
// ordinarylight/renderers/reference/path_tracer.py:55-65), gaining
// emission and single-scattered light and losing transmittance.
//
// From ordinarylight/volume/_core.py:
//   intersect_unit_boxes (:252-275)  slab test against the transformed unit
//                                    cube, entry clamped at 0;
//   sample_trilinear (:278-307)      trilinear lookup of the normalized grid
//                                    at clip(local, 0, 1) * (size - 1);
//   _volume_transfer_sample (:33-44) the RGBA transfer function (clamp,
//                                    repeat or mirror; linear or nearest),
//                                    missing values mapped to its entry 0;
//   volume_clip_mask (:310-318)      half-spaces (a, b, c) . p >= d - 1e-6;
//   _approximate_light_transmittance (:150-180)  one midpoint extinction
//                                    sample per medium towards the light;
//   _point_light_scattering (:183-249)  phase-weighted analytic-light
//                                    radiance, higher orders by the trapping
//                                    ratio, times the scattering colour;
//   integrate_volumes (:396-504)     the scattering source of each medium at
//                                    its interval midpoint, then a march over
//                                    the segments between interval events at
//                                    the smallest active step size (at most
//                                    4,096 steps), extinctions of overlapping
//                                    media added, emission weighted by
//                                    extinction, ending below transmittance
//                                    1e-4.
// Accumulation is in float32 (the reference sums in float64); the march is a
// deterministic quadrature, so the difference stays at float rounding.
#pragma once

#include "olc_common.cuh"

namespace olc {

constexpr uint32_t kMaxRefVolumes = 8;   // visible volumes per scene
constexpr uint32_t kMaxRefSteps = 4096;  // steps per segment (integrate_volumes)

OLC_D float3 rv_apply(const RefVolume& v, float3 p) {
  return f3(dot(f3(v.w2b0), p) + v.w2b0.w, dot(f3(v.w2b1), p) + v.w2b1.w, dot(f3(v.w2b2), p) + v.w2b2.w);
}
OLC_D float3 rv_linear(const RefVolume& v, float3 d) { return f3(dot(f3(v.w2b0), d), dot(f3(v.w2b1), d), dot(f3(v.w2b2), d)); }

// Entry and exit distances of the ray in the volume's unit cube; false when
// it misses (exit < max(entry, 0)).
OLC_D bool rv_box(const RefVolume& v, float3 o, float3 d, float& entry, float& leave) {
  const float3 lo = rv_apply(v, o), ld = rv_linear(v, d);
  const float l[3] = {lo.x, lo.y, lo.z}, dd[3] = {ld.x, ld.y, ld.z};
  float en = -CUDART_INF_F, ex = CUDART_INF_F;
  for (int a = 0; a < 3; ++a) {
    const float safe = fabsf(dd[a]) > 1e-12f ? dd[a] : copysignf(1e-12f, dd[a] + 1e-30f);
    const float t0 = -l[a] / safe, t1 = (1.0f - l[a]) / safe;
    en = fmaxf(en, fminf(t0, t1));
    ex = fminf(ex, fmaxf(t0, t1));
  }
  if (!(ex >= fmaxf(en, 0.0f))) return false;
  entry = fmaxf(en, 0.0f);
  leave = ex;
  return true;
}

OLC_D float rv_trilinear(const RefVolume& v, const float* grid, float3 p) {
  const float3 lp = rv_apply(v, p);
  const float c[3] = {clampf(lp.x, 0.0f, 1.0f) * (float)(v.nx - 1u), clampf(lp.y, 0.0f, 1.0f) * (float)(v.ny - 1u),
                      clampf(lp.z, 0.0f, 1.0f) * (float)(v.nz - 1u)};
  const uint32_t n[3] = {v.nx, v.ny, v.nz};
  uint32_t lo[3], hi[3];
  float w[3];
  for (int a = 0; a < 3; ++a) {
    const float f = floorf(c[a]);
    lo[a] = (uint32_t)f;
    hi[a] = min(lo[a] + 1u, n[a] - 1u);
    w[a] = c[a] - f;
  }
  const float* g = grid + v.grid_off;
  auto at = [&](uint32_t x, uint32_t y, uint32_t z) { return __ldg(g + ((uint64_t)z * v.ny + y) * v.nx + x); };
  const float c00 = at(lo[0], lo[1], lo[2]) * (1.0f - w[0]) + at(hi[0], lo[1], lo[2]) * w[0];
  const float c10 = at(lo[0], hi[1], lo[2]) * (1.0f - w[0]) + at(hi[0], hi[1], lo[2]) * w[0];
  const float c01 = at(lo[0], lo[1], hi[2]) * (1.0f - w[0]) + at(hi[0], lo[1], hi[2]) * w[0];
  const float c11 = at(lo[0], hi[1], hi[2]) * (1.0f - w[0]) + at(hi[0], hi[1], hi[2]) * w[0];
  const float c0 = c00 * (1.0f - w[1]) + c10 * w[1];
  const float c1 = c01 * (1.0f - w[1]) + c11 * w[1];
  return c0 * (1.0f - w[2]) + c1 * w[2];
}

OLC_D float4 rv_lut(const RefVolume& v, const float4* lut, float x) {
  float a;
  if (v.address == 0u) {
    a = clampf(x, 0.0f, 1.0f);
  } else if (v.address == 1u) {
    a = x - floorf(x);
  } else {
    float period = x - 2.0f * floorf(x * 0.5f);
    a = period <= 1.0f ? period : 2.0f - period;
  }
  const float pos = a * (float)(v.lut_len - 1u);
  const float4* t = lut + v.lut_off;
  if (!v.linear) return __ldg(t + min((uint32_t)floorf(pos + 0.5f), v.lut_len - 1u));
  const float f = floorf(pos);
  const uint32_t lo = min((uint32_t)f, v.lut_len - 1u), hi = min(lo + 1u, v.lut_len - 1u);
  const float w = pos - f;
  const float4 p = __ldg(t + lo), q = __ldg(t + hi);
  return make_float4(p.x * (1.0f - w) + q.x * w, p.y * (1.0f - w) + q.y * w, p.z * (1.0f - w) + q.z * w,
                     p.w * (1.0f - w) + q.w * w);
}

// Transfer-function sample of the value at p (zero where clipped away).
OLC_D float4 rv_rgba(const RefVolume& v, const float* grid, const float4* lut, float3 p) {
  for (uint32_t k = 0; k < v.num_clip; ++k)
    if (dot(f3(v.clip[k]), p) < v.clip[k].w - 1e-6f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float s = rv_trilinear(v, grid, p);
  if (v.missing) {
    const bool ok = isfinite(s);
    const float count = (float)v.lut_len;
    s = ok ? (1.0f + s * fmaxf(count - 2.0f, 0.0f)) / fmaxf(count - 1.0f, 1.0f) : 0.0f;
  }
  return rv_lut(v, lut, s);
}

OLC_D float rv_extinction(const RefVolume& v, float alpha_raw) {
  const float a = clampf(alpha_raw * v.density_scale, 0.0f, 1.0f - 1e-7f);
  return -log1pf(-a) / v.step_size;
}

struct RefVolumeView {
  const RefVolume* vols;
  uint32_t count;
  const float* grid;
  const float4* lut;
};

OLC_D RefVolumeView ref_volumes_of(const SceneRec& sc) {
  return RefVolumeView{sc.ref_vols, sc.num_ref_vols, sc.ref_grid, sc.ref_lut};
}

// Transmittance from p towards light_pos, one midpoint sample per medium.
OLC_D float rv_light_transmittance(const RefVolumeView& V, float3 p, float3 light_pos) {
  const float3 off = light_pos - p;
  const float dist = length(off);
  const float3 dir = off / fmaxf(dist, 1e-8f);
  float depth = 0.0f;
  for (uint32_t k = 0; k < V.count; ++k) {
    const RefVolume& v = V.vols[k];
    float en, ex;
    if (!rv_box(v, p, dir, en, ex)) continue;
    ex = fminf(ex, dist);
    if (!(ex > en)) continue;
    const float4 rgba = rv_rgba(v, V.grid, V.lut, p + dir * (0.5f * (en + ex)));
    depth += rv_extinction(v, rgba.w) * (ex - en);
  }
  return expf(-depth);
}

// Single-scattered analytic light at the medium point p seen along d
// (times the scattering colour; the caller scales by scattering_scale).
OLC_D float3 rv_scattering(const RefVolumeView& V, const RefVolume& v, const LightRec* lights, uint32_t num_lights,
                           float3 p, float3 d, float optical_depth) {
  float3 result = f3(0.0f, 0.0f, 0.0f), iso = f3(0.0f, 0.0f, 0.0f);
  const float g = v.scat_color_aniso.w;
  for (uint32_t i = 0; i < num_lights; ++i) {
    const LightRec L = lights[i];
    const int type = (int)(L.position_type.w + 0.5f);
    float3 incoming, light_pos;
    float atten = 1.0f;
    if (type == 1) {
      incoming = -normalize(f3(L.direction_range));
      light_pos = p + incoming * 10000.0f;
    } else {
      light_pos = f3(L.position_type);
      const float3 off = light_pos - p;
      const float d2 = fmaxf(dot(off, off), 1e-8f);
      const float dist = sqrtf(d2);
      incoming = off / dist;
      atten = 1.0f / d2;
      if (L.direction_range.w > 0.0f && dist > L.direction_range.w) atten = 0.0f;
      if (type == 2) {
        const float cone = dot(normalize(f3(L.direction_range)), -incoming);
        const float s = clampf((cone - L.spot.y) / fmaxf(L.spot.x - L.spot.y, 1e-8f), 0.0f, 1.0f);
        atten *= s * s * (3.0f - 2.0f * s);
      }
    }
    const float cosine = clampf(dot(incoming, d), -1.0f, 1.0f);
    float phase = 0.25f / OLC_PI_F;
    if (v.phase_hg) {
      const float den = fmaxf(1.0f + g * g - 2.0f * g * cosine, 1e-8f);
      phase = (1.0f - g * g) / (4.0f * OLC_PI_F * den * sqrtf(den));
    }
    const float3 incident =
        f3(L.color_intensity) * (L.color_intensity.w * atten * rv_light_transmittance(V, p, light_pos));
    result += incident * phase;
    iso += incident * (0.25f / OLC_PI_F);
  }
  if (v.orders > 1u) {
    const float trapping = 1.0f - expf(-fmaxf(optical_depth, 0.0f));
    const float3 ratio = f3(v.scat_albedo) * trapping;
    float3 power = ratio;
    for (uint32_t o = 2; o <= v.orders; ++o) {
      result += iso * power;
      power = power * ratio;
    }
  }
  return result * f3(v.scat_color_aniso);
}

// Radiance gained and transmittance of the segment [0, t_max] of the ray.
OLC_D void rv_integrate(const RefVolumeView& V, const LightRec* lights, uint32_t num_lights, float3 o, float3 d,
                        float t_max, float3& radiance, float& transmittance) {
  radiance = f3(0.0f, 0.0f, 0.0f);
  transmittance = 1.0f;
  float en[kMaxRefVolumes], ex[kMaxRefVolumes];
  float3 source[kMaxRefVolumes];
  uint32_t inside = 0;   // bit k: the ray crosses volume k
  float events[2 * kMaxRefVolumes];
  uint32_t ne = 0;
  for (uint32_t k = 0; k < V.count; ++k) {
    float a, b;
    if (!rv_box(V.vols[k], o, d, a, b)) continue;
    b = fminf(b, t_max);
    if (!(isfinite(a) && b > a)) continue;
    en[k] = a;
    ex[k] = b;
    inside |= 1u << k;
    const RefVolume& v = V.vols[k];
    source[k] = f3(0.0f, 0.0f, 0.0f);
    if (v.scattering_scale > 0.0f && num_lights > 0u) {
      const float3 mid = o + d * (0.5f * (a + b));
      const float4 rgba = rv_rgba(v, V.grid, V.lut, mid);
      const float depth = rv_extinction(v, rgba.w) * (b - a);
      source[k] = rv_scattering(V, v, lights, num_lights, mid, d, depth) * v.scattering_scale;
    }
    // events: sorted, without duplicates
    for (float e : {a, b}) {
      uint32_t pos = 0;
      while (pos < ne && events[pos] < e) ++pos;
      if (pos < ne && events[pos] == e) continue;
      for (uint32_t q = ne; q > pos; --q) events[q] = events[q - 1];
      events[pos] = e;
      ++ne;
    }
  }
  if (!inside) return;
  float T = 1.0f;
  float3 L = f3(0.0f, 0.0f, 0.0f);
  for (uint32_t s = 0; s + 1 < ne && T >= 1e-4f; ++s) {
    const float s0 = events[s], s1 = events[s + 1], mid = 0.5f * (s0 + s1);
    uint32_t active = 0;
    float ref_step = CUDART_INF_F;
    for (uint32_t k = 0; k < V.count; ++k)
      if (((inside >> k) & 1u) && en[k] <= mid && mid < ex[k]) {
        active |= 1u << k;
        ref_step = fminf(ref_step, V.vols[k].step_size);
      }
    if (!active) continue;
    const uint32_t steps = min((uint32_t)ceilf((s1 - s0) / ref_step), kMaxRefSteps);
    const float dt = (s1 - s0) / (float)max(steps, 1u);
    for (uint32_t i = 0; i < steps; ++i) {
      const float3 p = o + d * (s0 + ((float)i + 0.5f) * dt);
      float ext = 0.0f;
      float3 emit = f3(0.0f, 0.0f, 0.0f), scat = f3(0.0f, 0.0f, 0.0f);
      for (uint32_t k = 0; k < V.count; ++k) {
        if (!((active >> k) & 1u)) continue;
        const RefVolume& v = V.vols[k];
        const float4 rgba = rv_rgba(v, V.grid, V.lut, p);
        const float e = rv_extinction(v, rgba.w);
        ext += e;
        emit += f3(rgba.x, rgba.y, rgba.z) * (e * v.emission_scale);
        scat += source[k] * e;
      }
      if (ext > 1e-12f) {
        const float alpha = 1.0f - expf(-ext * dt);
        L += (emit + scat) * (T * alpha / ext);
        T *= 1.0f - alpha;
      }
      if (T < 1e-4f) break;
    }
  }
  radiance = L;
  transmittance = T;
}

}  // namespace olc
