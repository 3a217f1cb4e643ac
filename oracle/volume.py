"""ORACLE — test infrastructure only, never part of the product path.

numpy restatement of the participating-medium transport for parity tests of
the CUDA delta tracking:

* ``sample_trilinear`` restates the reference's dense-grid lookup
  (ordinarylight/volume/_core.py:271-307): local box coordinates clipped to
  [0, 1] and scaled by (n - 1), trilinear over the (z, y, x) grid;
* ``box_interval`` restates intersect_unit_boxes (:247-269) for one box;
* ``transmittance`` integrates exp(-sigma_t_scale * int density) by the
  midpoint rule with many steps (the reference ray-marches its media the same
  way, integrate_volume :323-395) — with a constant grid it is the analytic
  exp(-sigma_t d);
* ``render_medium`` is an independent Monte Carlo estimator of a scene made
  of the medium alone, lit by a constant environment and one directional
  light: delta-tracked free flights, isotropic scattering with a constant
  albedo, next-event estimation of the light through the exact
  transmittance, and the path-length rule of the CUDA renderer (vertex b
  samples the light and continues only while b + 1 < max_bounces).  Its
  random numbers are numpy's, so it agrees with the CUDA image in
  expectation, not bit for bit.
"""

from __future__ import annotations

import numpy as np

PI = 3.14159265358979


def sample_trilinear(grid, local):
    """Density at box-local points (..., 3) of a (z, y, x) grid."""
    grid = np.asarray(grid, np.float32)
    local = np.asarray(local, np.float64)
    shape_xyz = np.asarray(grid.shape[::-1], np.float64)
    c = np.clip(local, 0.0, 1.0) * (shape_xyz - 1.0)
    lo = np.floor(c).astype(np.int64)
    hi = np.minimum(lo + 1, np.asarray(grid.shape[::-1]) - 1)
    w = c - lo
    x0, y0, z0 = lo[..., 0], lo[..., 1], lo[..., 2]
    x1, y1, z1 = hi[..., 0], hi[..., 1], hi[..., 2]
    wx, wy, wz = w[..., 0], w[..., 1], w[..., 2]
    g = grid.astype(np.float64)
    c00 = g[z0, y0, x0] * (1 - wx) + g[z0, y0, x1] * wx
    c10 = g[z0, y1, x0] * (1 - wx) + g[z0, y1, x1] * wx
    c01 = g[z1, y0, x0] * (1 - wx) + g[z1, y0, x1] * wx
    c11 = g[z1, y1, x0] * (1 - wx) + g[z1, y1, x1] * wx
    c0 = c00 * (1 - wy) + c10 * wy
    c1 = c01 * (1 - wy) + c11 * wy
    return c0 * (1 - wz) + c1 * wz


def to_box(w2b, points, vectors=False):
    w2b = np.asarray(w2b, np.float64).reshape(3, 4)
    p = np.asarray(points, np.float64) @ w2b[:, :3].T
    return p if vectors else p + w2b[:, 3]


def box_interval(ob, db):
    """Entry/exit parameters of box-space rays in [0, 1]^3 (nan-safe)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / db
        a = -ob * inv
        b = (1.0 - ob) * inv
    lo = np.nanmax(np.minimum(a, b), axis=-1)
    hi = np.nanmin(np.maximum(a, b), axis=-1)
    return lo, hi


def transmittance(grid, w2b, sigma_scale, o, d, t_max=np.inf, steps=256, chunk=4096):
    """exp(-optical depth) of rays o + t d on (0, t_max): midpoint rule with
    `steps` equal steps over each ray's interval inside the box."""
    o = np.atleast_2d(np.asarray(o, np.float64))
    d = np.atleast_2d(np.asarray(d, np.float64))
    ob, db = to_box(w2b, o), to_box(w2b, d, vectors=True)
    t0, t1 = box_interval(ob, db)
    t0 = np.maximum(t0, 0.0)
    t1 = np.minimum(t1, t_max)
    out = np.ones(len(o))
    rows = np.flatnonzero(t1 > t0)
    frac = (np.arange(steps) + 0.5) / steps
    for start in range(0, rows.size, chunk):
        k = rows[start:start + chunk]
        length = t1[k] - t0[k]
        ts = t0[k, None] + frac[None, :] * length[:, None]
        dens = sample_trilinear(grid, ob[k, None, :] + ts[..., None] * db[k, None, :])
        out[k] = np.exp(-sigma_scale * dens.mean(axis=1) * length)
    return out


def _uniform_sphere(rng, n):
    z = 1.0 - 2.0 * rng.random(n)
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = 2.0 * PI * rng.random(n)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], -1)


def render_medium(grid, w2b, sigma_scale, albedo, origins, directions, *, env, light_dir=None, light_rgb=None,
                  max_bounces=4, seed=0, steps=128):
    """Radiance (n, 3) of the rays through a medium-only scene."""
    rng = np.random.default_rng(seed)
    grid = np.asarray(grid, np.float32)
    majorant = float(sigma_scale) * float(grid.max())
    o = np.asarray(origins, np.float64).copy()
    d = np.asarray(directions, np.float64).copy()
    n = len(o)
    rad = np.zeros((n, 3))
    tp = np.ones(n)
    alive = np.ones(n, bool)
    env = np.asarray(env, np.float64)
    if light_dir is not None:
        ldir = -np.asarray(light_dir, np.float64) / np.linalg.norm(light_dir)
        lrgb = np.asarray(light_rgb, np.float64)
    for bounce in range(max_bounces):
        idx = np.flatnonzero(alive)
        if idx.size == 0:
            break
        ob, db = to_box(w2b, o[idx]), to_box(w2b, d[idx], vectors=True)
        t0, t1 = box_interval(ob, db)
        t = np.maximum(t0, 0.0)
        inside = t1 > t
        collided = np.zeros(idx.size, bool)
        tc = np.zeros(idx.size)
        pending = inside.copy()
        while majorant > 0 and np.any(pending):
            p = np.flatnonzero(pending)
            t[p] -= np.log(1.0 - rng.random(p.size)) / majorant
            out = t[p] >= t1[p]
            pending[p[out]] = False
            q = p[~out]
            sigma = sigma_scale * sample_trilinear(grid, ob[q] + t[q, None] * db[q])
            real = rng.random(q.size) * majorant < sigma
            collided[q[real]] = True
            tc[q[real]] = t[q[real]]
            pending[q[real]] = False
        esc = idx[~collided]
        rad[esc] += tp[esc, None] * env
        alive[esc] = False
        hit = idx[collided]
        if hit.size == 0:
            continue
        pos = o[hit] + d[hit] * tc[collided, None]
        tp[hit] *= albedo
        if bounce + 1 >= max_bounces:
            alive[hit] = False
            continue
        if light_dir is not None:
            tr = transmittance(grid, w2b, sigma_scale, pos, np.broadcast_to(ldir, pos.shape), steps=steps)
            rad[hit] += (tp[hit] * tr / (4.0 * PI))[:, None] * lrgb
        o[hit] = pos
        d[hit] = _uniform_sphere(rng, hit.size)
    return rad


__all__ = ["sample_trilinear", "box_interval", "transmittance", "render_medium", "to_box"]
