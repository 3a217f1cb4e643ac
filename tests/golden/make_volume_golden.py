"""Generate reference-rendered fixtures for the reference-compatible
transport beyond the closed-box room, by running the REFERENCE's own
``CpuReferenceRenderer`` / ``ReferencePathTracer`` (imported like
make_golden.py does; ``--reference PATH`` or ``OL_REFERENCE_ROOT``):

* ``volume_small.npz``: the volume room of tests/parity_scenes.py (two
  overlapping media exercising the whole volume model) at 16 x 12, 2 spp,
  3 bounces, seed 1 — the oracle must reproduce it;
* ``compat_<case>.npz`` for the volume room (32 x 32, 3 bounces) and the
  scaled configs 2 and 3 of tests/parity_scenes.py (48 x 32, 4 bounces):
  independent batches of 64 samples (seeds 2000 and up; 64 batches, 4,096
  samples per pixel, where emitter fireflies make the noise heavy-tailed, 16
  for the terrain), their mean image, per-pixel standard error and per-batch
  image means.
* ``refpacked_scaled_terrain.npz``: the scaled config-3 scene built with the
  reference's own ``Scene`` API and flattened by this repository's packer,
  so a GPU test renders a scene that came from reference objects.

Run:  python tests/golden/make_volume_golden.py [--reference PATH] [--small-only]
"""

from __future__ import annotations

import multiprocessing as mp
import os
from pathlib import Path
import sys
import time

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path[:0] = [str(HERE), str(REPO), str(REPO / "tests")]

from make_golden import import_reference  # noqa: E402

BATCH_SPP = 64
BATCHES = {"volume_room": 64, "scaled_instanced": 64, "scaled_terrain": 16}
CONVERGED = {
    "volume_room": dict(size=(32, 32), max_bounces=3),
    "scaled_instanced": dict(size=(48, 32), max_bounces=4),
    "scaled_terrain": dict(size=(48, 32), max_bounces=4),
}


def _builder(name):
    import parity_scenes

    if name == "volume_room":
        return parity_scenes.volume_room
    return parity_scenes.COMPAT_CASES[name]["builder"]


def _batch(args):
    name, seed = args
    ol = import_reference()
    from ordinarylight.renderers.reference.path_tracer import ReferencePathTracer

    scene, camera = _builder(name)(ol)
    case = CONVERGED[name]
    w, h = case["size"]
    image = ReferencePathTracer(seed=seed).render_hdr(scene, camera, w, h, samples=BATCH_SPP,
                                                      max_bounces=case["max_bounces"])
    return image[..., :3].astype(np.float64)


def small():
    ol = import_reference()
    import parity_scenes
    from ordinarylight.renderers.reference.cpu import CpuReferenceRenderer

    scene, camera = parity_scenes.volume_room(ol)
    renderer = CpuReferenceRenderer(samples_per_pixel=2, max_bounces=3, seed=1)
    image = renderer.render_frame(scene, camera, 16, 12, frame_index=0)
    np.savez_compressed(HERE / "volume_small.npz", image=image, width=16, height=12, samples=2, max_bounces=3, seed=1)
    print("volume_small.npz written", flush=True)


def packed():
    ol = import_reference()
    import parity_scenes
    from ordinarylight_b200 import packing

    scene, _camera = parity_scenes.scaled_terrain(ol)
    packing.pack_scene(scene).save(HERE / "refpacked_scaled_terrain.npz")
    print("refpacked_scaled_terrain.npz written", flush=True)


def converged(name):
    t0 = time.time()
    batches = BATCHES[name]
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(os.cpu_count() or 1, batches)) as pool:
        images = pool.map(_batch, [(name, 2000 + k) for k in range(batches)])
    stack = np.stack(images)
    case = CONVERGED[name]
    w, h = case["size"]
    np.savez_compressed(HERE / f"compat_{name}.npz", mean=stack.mean(axis=0).astype(np.float32),
                        sem=(stack.std(axis=0, ddof=1) / np.sqrt(batches)).astype(np.float32),
                        batch_means=stack.reshape(batches, -1, 3).mean(axis=1), samples=batches * BATCH_SPP,
                        batches=batches, width=w, height=h, max_bounces=case["max_bounces"])
    print(f"compat_{name}.npz: {batches * BATCH_SPP} spp in {time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    small()
    packed()
    if "--small-only" not in sys.argv:
        names = [a for a in sys.argv[1:] if a in CONVERGED] or list(CONVERGED)
        for n in names:
            converged(n)
