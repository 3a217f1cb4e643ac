"""ORACLE — test infrastructure only, never part of the product path.

Restatement of the weighted-reservoir algebra of ReSTIR DI as the device
kernels apply it (ordinarylight_b200/csrc/olc_restir.cu: ``res_update``, the
temporal and spatial reuse of ``k_restir_initial`` / ``k_restir_spatial`` and
the contribution weight W written at finalisation), following the
reference's reservoir (ordinarylight/integrations/restir_di.py):

* streaming a candidate (``DirectLightReservoir.update``, restir_di.py:41-62):
  the count grows by the samples the candidate represents, the weight sum by
  its weight, and the candidate replaces the held sample when its weight is
  positive and either nothing is held yet or ``u * weight_sum < weight``
  (weight_sum already including it);
* reusing another reservoir (``merge``, restir_di.py:64-92): nothing happens
  for an empty source; otherwise the source's sample is streamed with weight
  ``target_here * source.weight_sum / source.target`` (0 when the source's
  target is not positive), the target re-evaluated at this surface, and the
  source's count as its represented samples;
* the contribution weight (``normalization``, restir_di.py:163-170):
  ``W = weight_sum / (count * target)``, 0 without a sample, a count or a
  positive target.

``dtype`` selects the arithmetic: ``np.float64`` is the reference's Python
float, ``np.float32`` the device's (every sum, product and quotient rounded
to float32, as the kernels compute them).  Candidate validation raises
``ValueError`` for the inputs the reference rejects.
"""

from __future__ import annotations

from dataclasses import dataclass
import math

import numpy as np

__all__ = ["Candidate", "Reservoir", "stream", "reuse", "cap_history", "contribution_weight"]


@dataclass(frozen=True)
class Candidate:
    """One light sample: emitter index, barycentrics, and its target value."""

    light: int
    u: float
    v: float
    target: float

    def __post_init__(self):
        if self.light < 0:
            raise ValueError("light cannot be negative")
        if not math.isfinite(self.target) or self.target < 0.0:
            raise ValueError("target must be finite and non-negative")


@dataclass
class Reservoir:
    """Held sample (None: empty), weight sum and represented sample count."""

    sample: Candidate | None = None
    weight_sum: float = 0.0
    count: int = 0


def stream(res: Reservoir, cand: Candidate, weight: float, random_value: float, *, represented: int = 1,
           dtype=np.float64) -> bool:
    """Stream one candidate; returns whether it is now the held sample."""
    if not math.isfinite(weight) or weight < 0.0:
        raise ValueError("weight must be finite and non-negative")
    if not 0.0 <= random_value < 1.0:
        raise ValueError("random value must lie in [0, 1)")
    if represented < 1:
        raise ValueError("a candidate represents at least one sample")
    w = dtype(weight)
    res.count += int(represented)
    res.weight_sum = dtype(dtype(res.weight_sum) + w)
    take = bool(w > 0.0) and (res.sample is None or bool(dtype(dtype(random_value) * res.weight_sum) < w))
    if take:
        res.sample = cand
    return take


def reuse(res: Reservoir, source: Reservoir, target_here: float, random_value: float, *, dtype=np.float64) -> bool:
    """Reuse `source` at this surface, its sample's target re-evaluated here."""
    if source.sample is None or source.count == 0:
        return False
    if not math.isfinite(target_here) or target_here < 0.0:
        raise ValueError("target at this surface must be finite and non-negative")
    t_here = dtype(target_here)
    t_src = dtype(source.sample.target)
    weight = dtype(dtype(t_here * dtype(source.weight_sum)) / t_src) if t_src > 0.0 else dtype(0.0)
    moved = Candidate(source.sample.light, source.sample.u, source.sample.v, float(t_here))
    return stream(res, moved, float(weight), random_value, represented=source.count, dtype=dtype)


def cap_history(source: Reservoir, cap: int, *, dtype=np.float64) -> Reservoir:
    """The previous frame's reservoir as temporal reuse sees it: its count
    clamped to `cap` and its weight sum scaled by (clamped / original), the
    history clamp of Bitterli et al., "Spatiotemporal reservoir resampling"
    (SIGGRAPH 2020), applied as the device does (``k_restir_initial``,
    cap = restir_max_history x candidates)."""
    if source.count <= 0:
        return Reservoir(source.sample, source.weight_sum, source.count)
    m = min(int(source.count), int(cap))
    scale = dtype(dtype(m) / dtype(source.count))
    return Reservoir(source.sample, float(dtype(dtype(source.weight_sum) * scale)), m)


def contribution_weight(res: Reservoir, *, dtype=np.float64) -> float:
    """W = weight_sum / (count * target); 0 without sample, count or target."""
    if res.sample is None or res.count == 0 or not res.sample.target > 0.0:
        return 0.0
    return float(dtype(dtype(res.weight_sum) / dtype(dtype(res.count) * dtype(res.sample.target))))
