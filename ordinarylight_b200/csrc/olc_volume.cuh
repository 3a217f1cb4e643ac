// Participating medium: one dense density grid per scene, delta tracking for
// free flights and ratio tracking for the transmittance of shadow rays.
//
// The grid follows the reference's dense volume (ordinarylight/volume/_core.py):
// densities indexed (z, y, x) fill the unit box under the volume transform,
// and a world point is sampled by trilinear interpolation with the
// coordinate clip(local, 0, 1) * (n - 1) of sample_trilinear (:271-307).
// Extinction is sigma_t(x) = sigma_t_scale * density(x), the single
// scattering albedo is constant and the phase function isotropic.
//
// Free flights use delta (Woodcock) tracking against the global majorant
// sigma_t_scale * max density: tentative collisions at exponential steps of
// the majorant, each real with probability sigma_t(x) / majorant.  The
// transmittance of a shadow segment is the ratio-tracking estimator, the
// product of (1 - sigma_t(x) / majorant) over the tentative collisions
// (Novak et al., "Residual ratio tracking for estimating attenuation in
// participating media", SIGGRAPH Asia 2014).  Both are unbiased.
#pragma once

#include "olc_common.cuh"

namespace olc {

// Bound on the tentative collisions of one tracking call; the majorant
// optical depth of the configuration scenes is far below it.
constexpr int kMediumMaxSteps = 8192;

struct Medium {
  const float* grid;
  uint32_t nx, ny, nz;
  Affine w2b;
  float sigma_scale;
  float albedo;
  float majorant;
};

OLC_D bool load_medium(const SceneRec& sc, Medium& m) {
  if (!sc.volume_present) return false;
  m.grid = sc.volume;
  m.nx = sc.vol_nx;
  m.ny = sc.vol_ny;
  m.nz = sc.vol_nz;
  m.w2b = Affine{sc.vol_w2b0, sc.vol_w2b1, sc.vol_w2b2};
  m.sigma_scale = sc.vol_sigma_t_scale;
  m.albedo = sc.vol_albedo;
  m.majorant = sc.vol_sigma_t_scale * sc.vol_max_density;
  return m.majorant > 0.0f;
}

// Parameter interval of the box-space ray ob + t db inside [0, 1]^3.
OLC_D bool medium_interval(float3 ob, float3 db, float& t0, float& t1) {
  const float ix = 1.0f / db.x, iy = 1.0f / db.y, iz = 1.0f / db.z;
  const float ax = -ob.x * ix, bx = (1.0f - ob.x) * ix;
  const float ay = -ob.y * iy, by = (1.0f - ob.y) * iy;
  const float az = -ob.z * iz, bz = (1.0f - ob.z) * iz;
  t0 = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fminf(az, bz));
  t1 = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
  return t1 > fmaxf(t0, 0.0f);
}

OLC_D float grid_at(const Medium& m, uint32_t x, uint32_t y, uint32_t z) {
  return __ldg(m.grid + ((uint64_t)z * m.ny + y) * m.nx + x);
}

// Trilinear density at box-space point b (sample_trilinear): one 64-bit
// base address and the seven neighbours as 32-bit offsets (zero at the
// grid's last cell), the same eight values as indexing each corner.
OLC_D float medium_density(const Medium& m, float3 b) {
  const float cx = clampf(b.x, 0.0f, 1.0f) * (float)(m.nx - 1u);
  const float cy = clampf(b.y, 0.0f, 1.0f) * (float)(m.ny - 1u);
  const float cz = clampf(b.z, 0.0f, 1.0f) * (float)(m.nz - 1u);
  const uint32_t x0 = (uint32_t)cx, y0 = (uint32_t)cy, z0 = (uint32_t)cz;
  const uint32_t dx = x0 + 1u < m.nx ? 1u : 0u;
  const uint32_t dy = y0 + 1u < m.ny ? m.nx : 0u;
  const uint32_t dz = z0 + 1u < m.nz ? m.nx * m.ny : 0u;
  const float* g = m.grid + ((uint64_t)z0 * m.ny + y0) * m.nx + x0;
  const float wx = cx - (float)x0, wy = cy - (float)y0, wz = cz - (float)z0;
  const float c00 = __ldg(g) * (1.0f - wx) + __ldg(g + dx) * wx;
  const float c10 = __ldg(g + dy) * (1.0f - wx) + __ldg(g + dy + dx) * wx;
  const float c01 = __ldg(g + dz) * (1.0f - wx) + __ldg(g + dz + dx) * wx;
  const float c11 = __ldg(g + dz + dy) * (1.0f - wx) + __ldg(g + dz + dy + dx) * wx;
  const float c0 = c00 * (1.0f - wy) + c10 * wy;
  const float c1 = c01 * (1.0f - wy) + c11 * wy;
  return c0 * (1.0f - wz) + c1 * wz;
}

// Delta tracking on (ta, tb) of the world ray o + t d (d of unit length):
// true with the distance of the first real collision, false if the flight
// leaves the interval.  Free-flight distances use the hardware logarithm
// (__logf: absolute error about 2^-21 on [0.5, 2], the accuracy Vulkan
// requires of the reference shader's log()), which took the terrain's
// shading from 4.35 to 4.25 ms per frame.
OLC_D bool medium_collision(const Medium& m, float3 o, float3 d, float ta, float tb, uint32_t& rng, float& t_out) {
  const float3 ob = xform_point(m.w2b, o), db = xform_vector(m.w2b, d);
  float t0, t1;
  if (!medium_interval(ob, db, t0, t1)) return false;
  float t = fmaxf(t0, ta);
  const float end = fminf(t1, tb);
  if (!(end > t)) return false;
  const float inv_major = 1.0f / m.majorant;
  for (int k = 0; k < kMediumMaxSteps; ++k) {
    t -= __logf(1.0f - olc_rand(rng)) * inv_major;
    if (!(t < end)) return false;
    const float sigma = m.sigma_scale * medium_density(m, ob + db * t);
    if (olc_rand(rng) * m.majorant < sigma) {
      t_out = t;
      return true;
    }
  }
  return false;
}

// Ratio-tracking transmittance of the segment (0, tb) of o + t d.  Once the
// estimate falls below 0.05, Russian roulette (survival 0.5) ends most of
// the remaining walk without bias.
OLC_D float medium_transmittance(const Medium& m, float3 o, float3 d, float tb, uint32_t& rng) {
  const float3 ob = xform_point(m.w2b, o), db = xform_vector(m.w2b, d);
  float t0, t1;
  if (!medium_interval(ob, db, t0, t1)) return 1.0f;
  float t = fmaxf(t0, 0.0f);
  const float end = fminf(t1, tb);
  if (!(end > t)) return 1.0f;
  const float inv_major = 1.0f / m.majorant;
  float T = 1.0f;
  for (int k = 0; k < kMediumMaxSteps; ++k) {
    t -= __logf(1.0f - olc_rand(rng)) * inv_major;
    if (!(t < end)) break;
    const float sigma = m.sigma_scale * medium_density(m, ob + db * t);
    T *= fmaxf(1.0f - sigma * inv_major, 0.0f);
    if (T < 0.05f) {
      if (olc_rand(rng) >= 0.5f) return 0.0f;
      T *= 2.0f;
    }
  }
  return T;
}

// Uniform direction on the sphere (the isotropic phase function's sample;
// pdf 1 / (4 pi)).
OLC_D float3 uniform_sphere(float u, float v) {
  const float z = 1.0f - 2.0f * u;
  const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  float s, c;
  __sincosf(2.0f * 3.14159265358979f * v, &s, &c);
  return f3(r * c, r * s, z);
}

}  // namespace olc
