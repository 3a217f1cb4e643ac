"""Generate tests/golden/analytic_lights.npz by running the REFERENCE's
analytic-light packing (Scene.analytic_light_data, scene/_core.py:2578-2632)
on a scene with point lights (with and without a range), directional lights
(unnormalised directions) and spot lights (ranges and cone angles), in that
interleaved order, without an environment.  The light parameters are stored
beside the records so the test builds the same lights.  Imports the
reference like make_golden.py does.

Run:  python tests/golden/make_light_golden.py
"""

from __future__ import annotations

from pathlib import Path
import sys

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import import_reference  # noqa: E402


def light_table(rng):
    """(kind, position, direction, color, intensity, range, inner, outer) rows;
    kind 0 point, 1 directional, 2 spot; range 0 means none."""
    rows = []
    for k in range(9):
        kind = k % 3
        pos = rng.uniform(-5.0, 5.0, 3)
        direction = rng.normal(size=3) * rng.uniform(0.2, 3.0)
        color = rng.uniform(0.0, 1.0, 3)
        intensity = float(rng.uniform(0.5, 50.0))
        rng_range = 0.0 if k in (0, 5) else float(rng.uniform(1.0, 20.0))
        inner = float(rng.uniform(0.0, 0.4))
        outer = float(inner + rng.uniform(0.05, 0.8))
        rows.append([kind, *pos, *direction, *color, intensity, rng_range, inner, outer])
    return np.asarray(rows, np.float64)


def build_lights(ol, table):
    lights = []
    for row in table:
        kind = int(row[0])
        pos, direction, color = tuple(row[1:4]), tuple(row[4:7]), tuple(row[7:10])
        intensity, rng_range, inner, outer = float(row[10]), float(row[11]), float(row[12]), float(row[13])
        rng_range = rng_range if rng_range > 0.0 else None
        if kind == 0:
            lights.append(ol.PointLight(position=pos, color=color, intensity=intensity, range=rng_range))
        elif kind == 1:
            lights.append(ol.DirectionalLight(direction=direction, color=color, intensity=intensity))
        else:
            lights.append(ol.SpotLight(position=pos, direction=direction, color=color, intensity=intensity,
                                       inner_cone_angle=inner, outer_cone_angle=outer, range=rng_range))
    return lights


def main():
    ol = import_reference()
    table = light_table(np.random.default_rng(77))
    scene = ol.Scene()
    for light in build_lights(ol, table):
        scene.add_light(light)
    records = np.asarray(scene.analytic_light_data(), np.float32)
    np.savez_compressed(HERE / "analytic_lights.npz", table=table, records=records)
    print(f"wrote analytic_lights.npz: {records.shape}")


if __name__ == "__main__":
    main()
