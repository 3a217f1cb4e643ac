"""ORACLE — test infrastructure only, never part of the product path.

numpy restatement of the reference GPU wavefront's dielectric interface
(wavefront_shade.comp:480-505) for scenes of flat-shaded transmissive
triangles under an equirect environment, where a path is deterministic:

* the interface normal faces the incoming ray (n, or -n when leaving);
* current IOR = top of the path's medium stack; target IOR = the material's
  max(ior, 1.0001) when entering, else the entry below the top (1 at the
  bottom); direction = GLSL refract(d, n, current / target), or
  reflect(d, n) on total internal reflection (|refract|^2 < 0.01);
* a refraction that enters pushes the target (up to the stack depth), one
  that leaves pops;
* throughput *= mix(1, base, 0.2) * transmission; the next ray starts 0.002
  along the new direction;
* a ray that leaves the scene adds throughput * environment(direction)
  (nearest texel, path_tracer.py:185-202) and ends; a path that reaches the
  bounce limit ends dark.

``trace`` also reports, per ray, whether every step stayed clear of
triangle edges, environment texel borders and the critical angle of total
internal reflection (where float rounding may pick the other side), so a
test compares only robust pixels.
"""

from __future__ import annotations

import numpy as np


def _hits(origins, dirs, tris, second=False):
    """Closest hit (t > 1e-4) of each ray by brute force: t, index, u, v
    (and, with second=True, the distance of the next-closest hit)."""
    n = len(origins)
    best_t = np.full(n, np.inf)
    next_t = np.full(n, np.inf)
    best = np.full(n, -1, np.int64)
    bu = np.zeros(n)
    bv = np.zeros(n)
    for k, tri in enumerate(tris):
        e1, e2 = tri[1] - tri[0], tri[2] - tri[0]
        p = np.cross(dirs, e2)
        det = p @ e1
        ok = np.abs(det) > 1e-12
        inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
        s = origins - tri[0]
        u = np.sum(s * p, axis=1) * inv
        q = np.cross(s, e1)
        v = np.sum(dirs * q, axis=1) * inv
        t = (q @ e2) * inv
        valid = ok & (u >= 0) & (v >= 0) & (u + v <= 1) & (t > 1e-4)
        hit = valid & (t < best_t)
        next_t = np.where(hit, best_t, np.where(valid, np.minimum(next_t, t), next_t))
        best_t[hit], best[hit], bu[hit], bv[hit] = t[hit], k, u[hit], v[hit]
    if second:
        return best_t, best, bu, bv, next_t
    return best_t, best, bu, bv


def _refract(d, n, eta, with_k=False):
    ni = np.sum(n * d, axis=1)
    k = 1.0 - eta * eta * (1.0 - ni * ni)
    out = eta[:, None] * d - (eta * ni + np.sqrt(np.maximum(k, 0.0)))[:, None] * n
    out[k < 0.0] = 0.0
    return (out, k) if with_k else out


def _environment(dirs, image, color, rotation, margin):
    lon = np.arctan2(dirs[:, 2], dirs[:, 0]) + rotation
    u = np.mod(lon / (2.0 * np.pi) + 0.5, 1.0)
    v = np.arccos(np.clip(dirs[:, 1], -1.0, 1.0)) / np.pi
    h, w, _ = image.shape
    fu, fv = u * w, v * h
    x = np.minimum(fu.astype(np.int64), w - 1)
    y = np.minimum(fv.astype(np.int64), h - 1)
    clear = (np.abs(fu - np.round(fu)) > margin) & (np.abs(fv - np.round(fv)) > margin)
    return image[y, x] * np.asarray(color), clear


def trace(origins, dirs, tris, transmission, ior, base, env_image, env_color=(1.0, 1.0, 1.0), env_rotation=0.0,
          max_bounces=16, max_depth=16, edge_margin=1e-3, texel_margin=2e-3, critical_margin=1e-3):
    """Radiance of each ray and whether its path is robust.  tris (N, 3, 3)
    world space; transmission, ior (N,) and base (N, 3) per triangle."""
    o = np.asarray(origins, np.float64).copy()
    d = np.asarray(dirs, np.float64).copy()
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tris = np.asarray(tris, np.float64)
    n_rays = len(o)
    radiance = np.zeros((n_rays, 3))
    tp = np.ones((n_rays, 3))
    stack = np.ones((n_rays, max_depth))
    depth = np.ones(n_rays, np.int64)
    alive = np.ones(n_rays, bool)
    robust = np.ones(n_rays, bool)
    ng_all = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    ng_all /= np.linalg.norm(ng_all, axis=1, keepdims=True)
    for bounce in range(max_bounces):
        idx = np.flatnonzero(alive)
        if not len(idx):
            break
        t, k, u, v, t2 = _hits(o[idx], d[idx], tris, second=True)
        gap = np.where(np.isfinite(t2), t2 - np.where(np.isfinite(t), t, 0.0), np.inf)
        robust[idx] &= (gap > 1e-4 * np.maximum(np.where(np.isfinite(t), t, 1.0), 1.0)) | (k < 0)   # no near-tie
        miss = k < 0
        if np.any(miss):
            mi = idx[miss]
            env, clear = _environment(d[mi], env_image, env_color, env_rotation, texel_margin)
            radiance[mi] += tp[mi] * env
            robust[mi] &= clear
            alive[mi] = False
        hi = idx[~miss]
        if not len(hi):
            break
        k, t, u, v = k[~miss], t[~miss], u[~miss], v[~miss]
        robust[hi] &= (u > edge_margin) & (v > edge_margin) & (1.0 - u - v > edge_margin)
        if bounce + 1 >= max_bounces:
            alive[hi] = False
            break
        ng = ng_all[k]
        di = d[hi]
        entering = np.sum(di * ng, axis=1) < 0.0
        nrm = np.where(entering[:, None], ng, -ng)
        dep = depth[hi]
        current = stack[hi, dep - 1]
        below = np.where(dep > 1, stack[hi, np.maximum(dep - 2, 0)], 1.0)
        target = np.where(entering, np.maximum(ior[k], 1.0001), below)
        w, k_disc = _refract(di, nrm, current / target, with_k=True)
        robust[hi] &= np.abs(k_disc) > critical_margin      # not at the critical angle
        tir = np.sum(w * w, axis=1) < 0.01
        w[tir] = di[tir] - 2.0 * np.sum(nrm[tir] * di[tir], axis=1)[:, None] * nrm[tir]
        push = ~tir & entering & (dep < max_depth)
        pop = ~tir & ~entering & (dep > 1)
        stack[hi[push], dep[push]] = target[push]
        depth[hi[push]] += 1
        depth[hi[pop]] -= 1
        tp[hi] *= (0.8 + 0.2 * base[k]) * transmission[k][:, None]
        w /= np.linalg.norm(w, axis=1, keepdims=True)
        p = o[hi] + di * t[:, None]
        o[hi] = p + w * 0.002
        d[hi] = w
    return radiance.astype(np.float32), robust
