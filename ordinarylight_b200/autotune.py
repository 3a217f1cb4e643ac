"""Launch-shape autotuner for batched rendering.

The wavefront's throughput depends on knobs that have no single best value
across workloads: the chunk size (paths resident per wavefront: small
chunks keep the working set in L2, large ones amortise launches and keep
every SM busy on the short queues of late bounces), the block shape of the
queue and traversal kernels, the traversal short-stack depth (shared memory
per thread against spills to local memory) and whether extension rays are
reordered by origin and direction before tracing (better shading coherence
on large scenes, at the cost of the reordering passes).  :func:`autotune`
times a given batch under candidate settings and leaves the renderer
configured with the fastest.  The search is coordinate descent (chunk size,
block shape, stack depth, ray reordering), 4 + 4 + 3 + 2 timed batches
instead of the 96 of the full grid; results are cached per workload
signature.

Changing these knobs never changes an image: the random numbers are keyed
per path and accumulation is order independent.
"""

from __future__ import annotations

from dataclasses import dataclass, field
import time

CHUNKS = (1 << 18, 1 << 20, 1 << 22, 1 << 24)
BLOCKS = ((64, 64), (128, 128), (256, 128), (512, 256))   # (queue kernels, traversal/shading)
STACKS = (16, 24, 32)
SORTS = (False, True)

_cache: dict = {}


@dataclass
class TuneResult:
    chunk_paths: int
    block_size: int
    trace_block: int
    stack_depth: int
    sort_rays: bool
    seconds: float
    trials: list = field(default_factory=list)


def workload_signature(requests) -> tuple:
    """Requests that plan alike: sizes, samples and bounce limits per scene."""
    return tuple(sorted((id(r.scene), int(r.width), int(r.height), r.samples, r.max_bounces) for r in requests))


def _time_batch(renderer, requests, outs, repeats: int) -> float:
    renderer.render_batch(requests, outs)      # warm-up (captures the graph)
    best = float("inf")
    for _ in range(repeats):
        t0 = time.perf_counter()
        renderer.render_batch(requests, outs)
        best = min(best, time.perf_counter() - t0)
    return best


def autotune(renderer, requests, *, chunks=CHUNKS, blocks=BLOCKS, stacks=STACKS, sorts=SORTS, repeats: int = 2,
             use_cache: bool = True) -> TuneResult:
    """Find the fastest (chunk_paths, block shape, stack_depth, ray
    reordering) for ``renderer.render_batch(requests)`` and apply it to the
    renderer."""
    requests = list(requests)
    key = (workload_signature(requests), renderer.config.mode, renderer.config.restir)
    if use_cache and key in _cache:
        result = _cache[key]
        renderer.reconfigure(chunk_paths=result.chunk_paths, block_size=result.block_size,
                             trace_block=result.trace_block, stack_depth=result.stack_depth,
                             sort_rays=result.sort_rays)
        return result
    import numpy as np

    outs = [np.empty((int(r.height), int(r.width), 4), np.float32) for r in requests]
    cfg = renderer.config
    current = {"chunk_paths": cfg.chunk_paths or chunks[-1], "block_size": cfg.block_size,
               "trace_block": cfg.trace_block, "stack_depth": cfg.stack_depth, "sort_rays": cfg.sort_rays}
    trials = []

    def trial(**changes):
        settings = dict(current, **changes)
        renderer.reconfigure(**settings)
        seconds = _time_batch(renderer, requests, outs, repeats)
        trials.append((settings, seconds))
        return seconds

    best = trial()
    for name, values in (("chunk_paths", [{"chunk_paths": c} for c in chunks]),
                         ("block", [{"block_size": b, "trace_block": t} for b, t in blocks]),
                         ("stack_depth", [{"stack_depth": s} for s in stacks]),
                         ("sort_rays", [{"sort_rays": bool(v)} for v in sorts])):
        choice = None
        for changes in values:
            if all(current.get(k) == v for k, v in changes.items()):
                continue
            seconds = trial(**changes)
            if seconds < best:
                best, choice = seconds, changes
        if choice:
            current.update(choice)
    renderer.reconfigure(**current)
    result = TuneResult(current["chunk_paths"], current["block_size"], current["trace_block"],
                        current["stack_depth"], current["sort_rays"], best, trials)
    _cache[key] = result
    return result


__all__ = ["autotune", "TuneResult", "workload_signature", "CHUNKS", "BLOCKS", "STACKS", "SORTS"]
