"""Generate tests/golden/reservoir.json by running the REFERENCE's reservoir
(ordinarylight/integrations/restir_di.py: DirectLightReservoir.update,
merge and normalization) on seeded candidate streams and reuse chains.
Imports the reference like make_golden.py does.

Each stream case lists its candidates (light, u, v, target, weight, random
value, represented samples) with the reference's per-candidate "selected"
answer and the final reservoir (light or -1, weight sum, count,
normalization).  Each reuse case builds a destination and several source
reservoirs from streams, then merges the sources in order (target at the
destination surface, random value) and records every merge's answer and the
final reservoir.

Run:  python tests/golden/make_reservoir_golden.py
"""

from __future__ import annotations

import json
from pathlib import Path
import sys

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import import_reference  # noqa: E402


def _candidates(rng, n, zero_fraction=0.2):
    out = []
    for _ in range(n):
        target = float(rng.lognormal(0.0, 1.5))
        weight = 0.0 if rng.random() < zero_fraction else float(target / rng.uniform(0.01, 2.0))
        represented = int(rng.integers(1, 4)) if rng.random() < 0.3 else 1
        out.append({"light": int(rng.integers(0, 1024)), "u": float(rng.random()), "v": float(rng.random()),
                    "target": target, "weight": weight, "random": float(rng.random()),
                    "represented": represented})
    return out


def _final(res):
    return {"light": -1 if res.sample is None else int(res.sample.light_index),
            "target": 0.0 if res.sample is None else float(res.sample.target),
            "weight_sum": float(res.weight_sum), "count": int(res.sample_count),
            "normalization": float(res.normalization)}


def _run_stream(mod, cands):
    res = mod.DirectLightReservoir()
    selected = []
    for c in cands:
        s = mod.DirectLightSample(c["light"], c["u"], c["v"], c["target"])
        selected.append(bool(res.update(s, c["weight"], c["random"], represented_samples=c["represented"])))
    return res, selected


def main():
    import_reference()
    from ordinarylight.integrations import restir_di as mod

    rng = np.random.default_rng(2024)
    streams = []
    for k in range(24):
        n = int(rng.integers(1, 33))
        cands = _candidates(rng, n, zero_fraction=0.0 if k == 0 else (1.0 if k == 1 else 0.2))
        res, selected = _run_stream(mod, cands)
        streams.append({"candidates": cands, "selected": selected, "final": _final(res)})

    reuses = []
    for k in range(24):
        dest_cands = _candidates(rng, int(rng.integers(0, 17)))
        dest, dest_selected = _run_stream(mod, dest_cands)
        sources = []
        merges = []
        for j in range(int(rng.integers(1, 6))):
            src_cands = _candidates(rng, int(rng.integers(0, 13)), zero_fraction=1.0 if j == 3 else 0.2)
            src, _ = _run_stream(mod, src_cands)
            sources.append({"candidates": src_cands, "final": _final(src)})
            target_here = 0.0 if rng.random() < 0.15 else float(rng.lognormal(0.0, 1.5))
            u = float(rng.random())
            merges.append({"source": j, "target_here": target_here, "random": u,
                           "reused": bool(dest.merge(src, target_here, u))})
        reuses.append({"destination": dest_cands, "destination_selected": dest_selected, "sources": sources,
                       "merges": merges, "final": _final(dest)})

    out = HERE / "reservoir.json"
    out.write_text(json.dumps({"streams": streams, "reuses": reuses}, separators=(",", ":")))
    print(f"wrote {out} ({out.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
