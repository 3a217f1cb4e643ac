"""ORACLE — test infrastructure only, never part of the product path.

numpy restatement of the reference GPU wavefront's isotropic PBR BSDF and
analytic-light terms (the CPU reference renderer has no GGX, so these are
pinned by the GLSL sources as specification):

* ``pbr_evaluate``  ordinarylight_pbr_evaluate
  (ordinarylight/shaders/ordinaryshade_primary.glsl:541-564):
  f0 = mix(0.04, base, metallic); F = f0 + (1 - f0)(1 - v.h)^5;
  alpha = max(roughness^2, 0.0009); D = a2 / (pi ((n.h)^2 (a2 - 1) + 1)^2)
  (uncapped: see _ggx_d);
  G1(x) = 2x / max(x + sqrt(a2 + (1 - a2) x^2), 1e-6);
  f = (1 - F)(1 - metallic) base / pi + F D G1(n.v) G1(n.l) / max(4 n.v n.l, 1e-6)
* ``pbr_pdf``       ordinarylight_pbr_pdf (:565-581)
* ``directional_radiance`` / ``point_radiance``: one analytic light's
  contribution f * color * intensity * attenuation * max(n.l, 0)
  (samplePointLights, transport_v1/lighting.glsl:260-312).
"""

from __future__ import annotations

import numpy as np

PI = 3.14159265358979


def _normalize(v):
    v = np.asarray(v, np.float64)
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def _ggx_d(n, h, nh, a2):
    """GGX D = a2 / (pi ((n.h)^2 (a2 - 1) + 1)^2), the bracket as
    |n x h|^2 + (n.h)^2 a2, uncapped (the reference's 1e-6 floor of pi den^2
    caps D near its peak below roughness 0.155, where its sampler still draws
    the uncapped distribution; above it both are the same function)."""
    c = np.cross(n, h)
    s2 = np.where(nh > 0.0, np.sum(c * c, -1), 1.0)
    den = s2 + nh * nh * a2
    return a2 / np.maximum(PI * den * den, 1e-300)


def pbr_evaluate(base, roughness, metallic, n, view, out):
    """roughness and metallic: scalars or one value per point."""
    base = np.asarray(base, np.float64)
    roughness = np.asarray(roughness, np.float64)
    metallic = np.asarray(metallic, np.float64)
    if metallic.ndim:
        metallic = metallic[..., None]
    n, view, out = _normalize(n), _normalize(view), _normalize(out)
    nv = np.maximum(np.sum(n * view, -1), 0.0)
    nl = np.maximum(np.sum(n * out, -1), 0.0)
    h = _normalize(view + out)
    nh = np.maximum(np.sum(n * h, -1), 0.0)
    vh = np.maximum(np.sum(view * h, -1), 0.0)
    f0 = 0.04 + (base - 0.04) * metallic
    w = (1.0 - np.clip(vh, 0.0, 1.0)) ** 5
    F = f0 + (1.0 - f0) * w[..., None]
    a = np.maximum(roughness * roughness, 0.0009)
    a2 = a * a
    D = _ggx_d(n, h, nh, a2)

    def g1(x):
        return 2.0 * x / np.maximum(x + np.sqrt(a2 + (1.0 - a2) * x * x), 1e-6)

    G = g1(nv) * g1(nl)
    spec = F * (D * G / np.maximum(4.0 * nv * nl, 1e-6))[..., None]
    diff = (1.0 - F) * (1.0 - metallic) * base / PI
    f = diff + spec
    valid = (nv > 0.0) & (nl > 0.0)
    return np.where(valid[..., None], f, 0.0)


def pbr_pdf(base, roughness, metallic, n, view, out):
    base = np.asarray(base, np.float64)
    n, view, out = _normalize(n), _normalize(view), _normalize(out)
    nl = np.maximum(np.sum(n * out, -1), 0.0)
    h = _normalize(view + out)
    nh = np.maximum(np.sum(n * h, -1), 0.0)
    vh = np.maximum(np.sum(view * h, -1), 1e-6)
    a = max(roughness * roughness, 0.0009)
    a2 = a * a
    spec_pdf = _ggx_d(n, h, nh, a2) * nh / (4.0 * vh)
    diff_pdf = nl / PI
    f0 = 0.04 + (base - 0.04) * metallic
    p = np.clip(np.max(f0), 0.1, 0.9)
    return np.where(nl > 0.0, diff_pdf + (spec_pdf - diff_pdf) * p, 0.0)


def directional_radiance(base, roughness, metallic, n, view, light_direction, color, intensity):
    """Radiance reflected towards ``view`` from one directional light shining
    along ``light_direction``."""
    l = -_normalize(light_direction)
    l = np.broadcast_to(l, np.shape(n))
    f = pbr_evaluate(base, roughness, metallic, n, view, l)
    cos = np.maximum(np.sum(_normalize(n) * l, -1), 0.0)
    return f * np.asarray(color, np.float64) * intensity * cos[..., None]


def point_radiance(base, roughness, metallic, p, n, view, light_position, color, intensity):
    off = np.asarray(light_position, np.float64) - np.asarray(p, np.float64)
    d2 = np.maximum(np.sum(off * off, -1), 1e-6)
    l = off / np.sqrt(d2)[..., None]
    f = pbr_evaluate(base, roughness, metallic, n, view, l)
    cos = np.maximum(np.sum(_normalize(n) * l, -1), 0.0)
    return f * np.asarray(color, np.float64) * intensity * (cos / d2)[..., None]
