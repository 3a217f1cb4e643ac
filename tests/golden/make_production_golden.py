"""Generate tests/golden/production_<case>.npz: converged images of the
production-estimator oracle (oracle/transport.c through oracle/production.py)
for the parity scenes of tests/parity_scenes.py.

Each fixture holds the per-pixel mean radiance (float32) and its standard
error (float16, from the per-sample variance), the oracle's settings and
seed, so tests/test_oracle_production.py can re-render any window and require
the same bits, and tests/test_gpu_production.py can compare the CUDA
renderer's production mode against it.  The oracle needs no reference
checkout.

Run:  python tests/golden/make_production_golden.py [case ...]
"""

from __future__ import annotations

from pathlib import Path
import sys
import time

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path[:0] = [str(REPO), str(REPO / "tests")]

import parity_scenes  # noqa: E402
from oracle import production  # noqa: E402

SEED = 1
SAMPLES = {"restir_spheres": 32768}
DEFAULT_SAMPLES = 8192


def make(name: str) -> None:
    case = parity_scenes.CASES[name]
    scene, camera = parity_scenes.build(name)
    w, h = case["size"]
    spp = SAMPLES.get(name, DEFAULT_SAMPLES)
    t0 = time.time()
    mean, sem = production.render(scene, camera, w, h, samples=spp, max_bounces=case["max_bounces"],
                                  rr_start=case["rr_start"], rr_min_survival=case["rr_min"],
                                  env_nee=case["env_nee"], seed=SEED)
    np.savez_compressed(HERE / f"production_{name}.npz", mean=mean.astype(np.float32), sem=sem.astype(np.float16),
                        samples=spp, seed=SEED, width=w, height=h, max_bounces=case["max_bounces"],
                        rr_start=case["rr_start"], rr_min=case["rr_min"], env_nee=case["env_nee"])
    print(f"{name}: {spp} spp in {time.time() - t0:.1f} s, mean {mean.mean(axis=(0, 1))}", flush=True)


if __name__ == "__main__":
    names = sys.argv[1:] or list(parity_scenes.CASES)
    for n in names:
        make(n)
