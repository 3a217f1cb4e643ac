"""Generate the golden fixtures of tests/golden/ by running the REFERENCE.

Imports OrdinaryLight from a reference checkout (read-only; ``--reference
PATH``, else the ``OL_REFERENCE_ROOT`` environment variable, else a
``reference`` directory beside this repository) with three stub
modules for its un-vendored dependencies (``ordinaryshade``, ``pygltflib`` and
the material compiler ``ordinarylight.materials.shade``, none of which the
CPU reference renderer uses), builds the benchmark scenes through the
reference's own ``ordinarylight.Scene`` API, and records what the reference
computes:

* ``config1_scene.npz``    Scene.triangles() soup of the closed-box room,
                           emissive_triangle_data(), emissive_light_weight
* ``config1_primary.npz``  256x256 camera rays of sample 0 (seed 1): SHA-256 of
                           the rays (float64 and rounded to float32) and
                           ReferencePathTracer._intersect on the float32 rays
* ``config1_render_small.npz`` CpuReferenceRenderer images (24x16, 2 spp,
                           4 bounces, seed 1) at frame_index 0 and 3
* ``spheres_small.npz``    a 2-instance sphere scene: soup, emitter records,
                           camera rays and _intersect results
* ``config1_converged.npz`` 256x256, 4 bounces, 16 batches x 64 spp with
                           seeds 1000..1015: mean image and per-pixel
                           standard error of the mean
The reference is not available where the GPU tests run; these files are.

Run:  python tests/golden/make_golden.py [--reference PATH] [--skip-converged]
"""

from __future__ import annotations

import multiprocessing as mp
import os
from pathlib import Path
import sys
import time
import types

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def reference_root() -> Path:
    """The reference checkout: ``--reference PATH`` on the command line, else
    ``OL_REFERENCE_ROOT``, else ``reference`` beside this repository."""
    if "--reference" in sys.argv:
        return Path(sys.argv[sys.argv.index("--reference") + 1]).resolve()
    if os.environ.get("OL_REFERENCE_ROOT"):
        return Path(os.environ["OL_REFERENCE_ROOT"]).resolve()
    return REPO.parent / "reference"


def reference_available() -> bool:
    return (reference_root() / "ordinarylight" / "__init__.py").exists()


def import_reference():
    """Import the reference package with its three optional dependencies stubbed."""
    if "ordinarylight.renderers.reference.cpu" in sys.modules:
        import ordinarylight as ol

        return ol

    class _Permissive(types.ModuleType):
        def __getattr__(self, name):
            if name.startswith("__"):
                raise AttributeError(name)

            def anything(*_args, **_kwargs):
                return anything

            return anything

    sys.modules.setdefault("ordinaryshade", _Permissive("ordinaryshade"))
    sys.modules.setdefault("pygltflib", _Permissive("pygltflib"))
    shade = types.ModuleType("ordinarylight.materials.shade")
    shade.compile_material = lambda *a, **k: None
    shade.compile_dispatch = lambda *a, **k: None
    sys.modules["ordinarylight.materials.shade"] = shade
    root = reference_root()
    if not reference_available():
        raise RuntimeError(f"no OrdinaryLight checkout at {root}; pass --reference PATH or set OL_REFERENCE_ROOT")
    if str(root) not in sys.path:
        sys.path.insert(0, str(root))
    import ordinarylight as ol
    import ordinarylight.renderers.reference.cpu  # noqa: F401

    return ol


def _sha(array):
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def _scenes(ol):
    sys.path.insert(0, str(REPO))
    from ordinarylight_b200 import scenes

    return scenes


def _batch(args):
    seed, spp, width, height, bounces = args
    ol = import_reference()
    scenes = _scenes(ol)
    scene, camera = scenes.box_room(ol)
    from ordinarylight.renderers.reference.path_tracer import ReferencePathTracer

    image = ReferencePathTracer(seed=seed).render_hdr(scene, camera, width, height, samples=spp,
                                                      max_bounces=bounces)
    return image[..., :3].astype(np.float64)


def main(skip_converged=False):
    ol = import_reference()
    scenes = _scenes(ol)
    from ordinarylight.renderers.reference.cpu import CpuReferenceRenderer
    from ordinarylight.renderers.reference.path_tracer import ReferencePathTracer

    scene, camera = scenes.box_room(ol)
    tris, colors, emissions = scene.triangles()
    np.savez_compressed(HERE / "config1_scene.npz", triangles=tris, colors=colors, emissions=emissions,
                        emitters=scene.emissive_triangle_data(), emissive_weight=scene.emissive_light_weight,
                        instance_ids=scene.triangle_instance_ids())

    rng = np.random.default_rng(1)
    origins, directions = ReferencePathTracer._camera_rays(camera, 256, 256, rng)
    o32 = origins.astype(np.float32)
    d32 = directions.astype(np.float32)
    t, tri = ReferencePathTracer._intersect(o32, d32, tris)
    np.savez_compressed(HERE / "config1_primary.npz", origins_sha256=_sha(o32), directions_sha256=_sha(d32),
                        directions_f64_sha256=_sha(np.ascontiguousarray(directions)), t=t,
                        triangle=tri.astype(np.int16), width=256, height=256, seed=1)

    renderer = CpuReferenceRenderer(samples_per_pixel=2, max_bounces=4, seed=1)
    img0 = renderer.render_frame(scene, camera, 24, 16, frame_index=0)
    img3 = renderer.render_frame(scene, camera, 24, 16, frame_index=3)
    np.savez_compressed(HERE / "config1_render_small.npz", frame0=img0, frame3=img3, width=24, height=16,
                        samples=2, max_bounces=4, seed=1)

    sscene, scamera = scenes.instanced_spheres(ol, seed=5, instances=2, segments=16, bands=9, emitters=4,
                                               extent=3.0)
    stris, _c, _e = sscene.triangles()
    srng = np.random.default_rng(9)
    so, sd = ReferencePathTracer._camera_rays(scamera, 48, 32, srng)
    so32, sd32 = so.astype(np.float32), sd.astype(np.float32)
    st, stri = ReferencePathTracer._intersect(so32, sd32, stris)
    np.savez_compressed(HERE / "spheres_small.npz", triangles=stris, emitters=sscene.emissive_triangle_data(),
                        emissive_weight=sscene.emissive_light_weight, instance_ids=sscene.triangle_instance_ids(),
                        origins=so32, directions=sd32, t=st, triangle=stri)
    print("small fixtures written", flush=True)

    if skip_converged:
        return
    batches, spp = 16, 64
    t0 = time.time()
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(os.cpu_count() or 1, batches)) as pool:
        images = pool.map(_batch, [(1000 + k, spp, 256, 256, 4) for k in range(batches)])
    stack = np.stack(images)
    mean = stack.mean(axis=0)
    sem = stack.std(axis=0, ddof=1) / np.sqrt(batches)
    np.savez_compressed(HERE / "config1_converged.npz", mean=mean.astype(np.float32), sem=sem.astype(np.float32),
                        batch_means=stack.reshape(batches, -1, 3).mean(axis=1).astype(np.float64),
                        samples=batches * spp, batches=batches, width=256, height=256, max_bounces=4)
    print(f"converged fixture: {batches * spp} spp in {time.time() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main(skip_converged="--skip-converged" in sys.argv)
