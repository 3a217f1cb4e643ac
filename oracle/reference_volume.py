"""ORACLE — test infrastructure only, never part of the product path.

numpy restatement of the reference CPU renderer's volume model, the
emission–absorption ray march with point-light single scattering that
``ReferencePathTracer.render_hdr`` applies to every ray segment
(ordinarylight/renderers/reference/path_tracer.py:55-65) — from
ordinarylight/volume/_core.py:

* ``intersect_unit_boxes`` (:252-275): slab test of the ray against each
  volume's transformed local unit cube; entry clamped at 0, misses (inf, -inf);
* ``sample_trilinear`` (:278-307): trilinear lookup of the normalized grid
  (z, y, x) at clip(local, 0, 1) * (size - 1);
* ``transfer`` (``_volume_transfer_sample``, :33-44, and ``Texture1D.sample``,
  scene/_core.py:168-186): the RGBA lookup table addressed by clamp, repeat
  or mirror, linear or nearest, with the reserved first entry of
  missing-data volumes;
* ``clip_mask`` (:310-318): half-space clip planes with a 1e-6 margin;
* ``approximate_light_transmittance`` (:150-180): one midpoint extinction
  sample per crossed medium towards the light;
* ``point_light_scattering`` (:183-249): phase-weighted incident radiance of
  every analytic light (directional, point with range, spot with its
  smoothstep cone), multiple scattering orders by the trapping ratio,
  times the scattering colour;
* ``integrate_volumes`` (:396-504): per ray, each medium's scattering source
  at its interval midpoint, then a march over the segments between interval
  events (step = the smallest active step size, at most 4,096 steps), with
  the extinctions of overlapping media added and emission weighted by
  extinction, stopping below a transmittance of 1e-4.

The order of operations and the float32 / float64 types follow the
reference, so ``tests/golden/make_golden.py``'s reference renders of a volume
scene are reproduced (``tests/test_oracle_golden.py``).
"""

from __future__ import annotations

import numpy as np

_INV_4PI = 1.0 / (4.0 * np.pi)


def _inverse(volume):
    return np.linalg.inv(volume.transform.matrix).astype(np.float32)


def intersect_unit_boxes(origins, directions, volumes):
    origins = np.asarray(origins, np.float32)
    directions = np.asarray(directions, np.float32)
    entries = np.full((len(volumes), len(origins)), np.inf, np.float32)
    exits = np.full_like(entries, -np.inf)
    for index, volume in enumerate(volumes):
        inv = _inverse(volume)
        lo = origins @ inv[:3, :3].T + inv[:3, 3]
        ld = directions @ inv[:3, :3].T
        safe = np.where(np.abs(ld) > 1e-12, ld, np.copysign(1e-12, ld + 1e-30))
        a = -lo / safe
        b = (1.0 - lo) / safe
        entry = np.max(np.minimum(a, b), axis=1)
        leave = np.min(np.maximum(a, b), axis=1)
        valid = leave >= np.maximum(entry, 0.0)
        entries[index, valid] = np.maximum(entry[valid], 0.0)
        exits[index, valid] = leave[valid]
    return entries, exits


def sample_trilinear(volume, world_positions):
    positions = np.asarray(world_positions, np.float32)
    inv = _inverse(volume)
    local = positions @ inv[:3, :3].T + inv[:3, 3]
    shape_xyz = np.asarray(volume.data.shape[::-1], np.float32)
    coords = np.clip(local, 0.0, 1.0) * (shape_xyz - 1.0)
    lower = np.floor(coords).astype(np.int64)
    upper = np.minimum(lower + 1, np.asarray(volume.data.shape[::-1]) - 1)
    w = coords - lower
    x0, y0, z0 = lower.T
    x1, y1, z1 = upper.T
    wx, wy, wz = w.T
    g = volume.normalized_data
    c00 = g[z0, y0, x0] * (1.0 - wx) + g[z0, y0, x1] * wx
    c10 = g[z0, y1, x0] * (1.0 - wx) + g[z0, y1, x1] * wx
    c01 = g[z1, y0, x0] * (1.0 - wx) + g[z1, y0, x1] * wx
    c11 = g[z1, y1, x0] * (1.0 - wx) + g[z1, y1, x1] * wx
    c0 = c00 * (1.0 - wy) + c10 * wy
    c1 = c01 * (1.0 - wy) + c11 * wy
    return np.asarray(c0 * (1.0 - wz) + c1 * wz, np.float32)


def lut_sample(values, address_mode, linear, coordinates):
    """A 1D RGBA lookup table at normalized coordinates."""
    values = np.asarray(values, np.float32)
    x = np.asarray(coordinates, np.float32)
    if address_mode == "clamp":
        a = np.clip(x, 0.0, 1.0)
    elif address_mode == "repeat":
        a = x - np.floor(x)
    else:
        period = np.mod(x, 2.0)
        a = np.where(period <= 1.0, period, 2.0 - period)
    position = a * max(len(values) - 1, 0)
    if not linear:
        return np.asarray(values[np.floor(position + 0.5).astype(np.int64)], np.float32)
    lo = np.floor(position).astype(np.int64)
    hi = np.minimum(lo + 1, len(values) - 1)
    w = (position - lo)[..., None]
    return np.asarray(values[lo] * (1.0 - w) + values[hi] * w, np.float32)


def transfer(volume, scalars):
    tf = volume.material.transfer_function
    scalars = np.asarray(scalars, np.float32)
    if not volume.missing_data:
        return lut_sample(tf.values, tf.address_mode, tf.linear_filter, scalars)
    valid = np.isfinite(scalars)
    count = len(tf.values)
    encoded = (1.0 + np.where(valid, scalars, 0.0) * max(count - 2, 0)) / max(count - 1, 1)
    return lut_sample(tf.values, tf.address_mode, tf.linear_filter, np.where(valid, encoded, 0.0))


def clip_mask(volume, world_positions):
    positions = np.asarray(world_positions, np.float32)
    keep = np.ones(len(positions), bool)
    for plane in volume.clip_planes:
        keep &= positions @ np.asarray(plane[:3], np.float32) >= float(plane[3]) - 1e-6
    return keep


def _phase(cosine, material):
    cosine = np.clip(np.asarray(cosine, np.float32), -1.0, 1.0)
    if material.phase_function == "isotropic":
        return np.full_like(cosine, _INV_4PI, dtype=np.float32)
    g = float(material.anisotropy)
    den = np.maximum(1.0 + g * g - 2.0 * g * cosine, 1e-8)
    return np.asarray((1.0 - g * g) / (4.0 * np.pi * den ** 1.5), np.float32)


def _extinction(volume, positions):
    rgba = transfer(volume, sample_trilinear(volume, positions))
    rgba[~clip_mask(volume, positions)] = 0.0
    alpha = np.clip(rgba[:, 3] * volume.material.density_scale, 0.0, 1.0 - 1e-7)
    return -np.log1p(-alpha) / volume.material.step_size


def approximate_light_transmittance(volumes, positions, light_position):
    if not volumes:
        return np.ones(len(positions), np.float32)
    offset = np.asarray(light_position, np.float32) - positions
    distance = np.linalg.norm(offset, axis=1)
    dirs = offset / np.maximum(distance, 1e-8)[:, None]
    entries, exits = intersect_unit_boxes(positions, dirs, volumes)
    depth = np.zeros(len(positions), np.float32)
    for index, volume in enumerate(volumes):
        entry = np.maximum(entries[index], 0.0)
        leave = np.minimum(exits[index], distance)
        valid = np.isfinite(entry) & (leave > entry)
        if not np.any(valid):
            continue
        ids = np.flatnonzero(valid)
        mid = 0.5 * (entry[ids] + leave[ids])
        depth[ids] += _extinction(volume, positions[ids] + dirs[ids] * mid[:, None]) * (leave[ids] - entry[ids])
    return np.asarray(np.exp(-depth), np.float32)


def point_light_scattering(material, positions, view_directions, lights, volumes=(), optical_depth=None):
    if material.scattering_scale <= 0.0 or not lights:
        return np.zeros((len(positions), 3), np.float32)
    result = np.zeros((len(positions), 3), np.float32)
    isotropic = np.zeros_like(result)
    outgoing = -np.asarray(view_directions, np.float32)
    for light in lights:
        kind = type(light).__name__
        attenuation = np.ones(len(positions), np.float32)
        if kind == "DirectionalLight":
            incoming_dir = -np.asarray(light.direction, np.float32)
            incoming_dir /= np.linalg.norm(incoming_dir)
            incoming = np.repeat(incoming_dir[None, :], len(positions), axis=0)
            light_positions = positions + incoming * 10000.0
        else:
            light_position = np.asarray(light.position, np.float32)
            offset = light_position - positions
            d2 = np.maximum(np.sum(offset * offset, axis=1), 1e-8)
            distance = np.sqrt(d2)
            incoming = offset / distance[:, None]
            attenuation /= d2
            if light.range is not None:
                attenuation[distance > light.range] = 0.0
            if kind == "SpotLight":
                axis = np.asarray(light.direction, np.float32)
                axis /= np.linalg.norm(axis)
                cone = np.sum(axis[None, :] * -incoming, axis=1)
                inner, outer = np.cos(light.inner_cone_angle), np.cos(light.outer_cone_angle)
                spot = np.clip((cone - outer) / max(inner - outer, 1e-8), 0, 1)
                attenuation *= spot * spot * (3.0 - 2.0 * spot)
            light_positions = np.repeat(light_position[None, :], len(positions), axis=0)
        phase = _phase(np.sum(-incoming * outgoing, axis=1), material)
        incident = np.asarray(light.color, np.float32)[None, :] * float(light.intensity) * attenuation[:, None]
        incident *= approximate_light_transmittance(volumes, positions, light_positions)[:, None]
        result += incident * phase[:, None]
        isotropic += incident * _INV_4PI
    if material.scattering_orders > 1 and optical_depth is not None:
        trapping = 1.0 - np.exp(-np.maximum(np.asarray(optical_depth, np.float32), 0.0))
        ratio = trapping[:, None] * np.asarray(material.scattering_albedo, np.float32)[None, :]
        power = ratio.copy()
        for _order in range(2, material.scattering_orders + 1):
            result += isotropic * power
            power *= ratio
    return result * np.asarray(material.scattering_color, np.float32)[None, :]


def integrate_volumes(volumes, origins, directions, entries, exits, *, max_distance=None, lights=()):
    volumes = tuple(volumes)
    origins = np.asarray(origins, np.float32)
    directions = np.asarray(directions, np.float32)
    entries = np.asarray(entries, np.float32)
    exits = np.asarray(exits, np.float32)
    if max_distance is not None:
        exits = np.minimum(exits, np.asarray(max_distance, np.float32))
    radiance = np.zeros((len(origins), 3), np.float32)
    transmittance = np.ones(len(origins), np.float32)
    for r in range(len(origins)):
        intervals = []
        for v in range(len(volumes)):
            entry = float(max(entries[v, r], 0.0))
            leave = float(exits[v, r])
            if np.isfinite(entry) and leave > entry:
                intervals.append((entry, leave, v))
        if not intervals:
            continue
        events = sorted({e for iv in intervals for e in iv[:2]})
        ray_radiance = np.zeros(3, np.float64)
        ray_t = 1.0
        sources = {}
        for entry, leave, v in intervals:
            volume = volumes[v]
            mat = volume.material
            position = origins[r] + directions[r] * (0.5 * (entry + leave))
            rgba = transfer(volume, sample_trilinear(volume, position[None, :]))[0]
            if not clip_mask(volume, position[None, :])[0]:
                rgba = np.zeros(4, np.float32)
            alpha = float(np.clip(rgba[3] * mat.density_scale, 0.0, 1.0 - 1e-7))
            depth = np.asarray((-np.log1p(-alpha) / mat.step_size * (leave - entry),), np.float32)
            sources[v] = point_light_scattering(mat, position[None, :], directions[r][None, :], lights, volumes,
                                                depth)[0] * mat.scattering_scale
        for s0, s1 in zip(events[:-1], events[1:]):
            mid = 0.5 * (s0 + s1)
            active = [v for entry, leave, v in intervals if entry <= mid < leave]
            if not active:
                continue
            ref_step = min(volumes[v].material.step_size for v in active)
            steps = min(int(np.ceil((s1 - s0) / ref_step)), 4096)
            dt = (s1 - s0) / max(steps, 1)
            for k in range(steps):
                position = origins[r] + directions[r] * (s0 + (k + 0.5) * dt)
                extinction = 0.0
                emission = np.zeros(3, np.float64)
                scattering = np.zeros(3, np.float64)
                for v in active:
                    volume = volumes[v]
                    mat = volume.material
                    rgba = transfer(volume, sample_trilinear(volume, position[None, :]))[0]
                    if not clip_mask(volume, position[None, :])[0]:
                        rgba = np.zeros(4, np.float32)
                    alpha = float(np.clip(rgba[3] * mat.density_scale, 0.0, 1.0 - 1e-7))
                    e = -np.log1p(-alpha) / mat.step_size
                    extinction += e
                    emission += e * rgba[:3] * mat.emission_scale
                    scattering += e * sources[v]
                if extinction > 1e-12:
                    a = 1.0 - np.exp(-extinction * dt)
                    ray_radiance += ray_t * a * (emission + scattering) / extinction
                    ray_t *= 1.0 - a
                if ray_t < 1e-4:
                    break
            if ray_t < 1e-4:
                break
        radiance[r] = ray_radiance
        transmittance[r] = ray_t
    return radiance, transmittance


__all__ = ["intersect_unit_boxes", "sample_trilinear", "lut_sample", "transfer", "clip_mask",
           "approximate_light_transmittance", "point_light_scattering", "integrate_volumes"]
