"""One frame's samples rendered across GPUs, one process per GPU.

The path shards without exchange: every sample of every pixel is an
independent path whose random numbers are keyed by (pixel, sample, bounce,
seed + frame_index).  Rank r of N renders the contiguous sample range
:func:`sample_shard` gives it, as one job whose ``first_sample`` is the start
of the range, and returns the job's unsigned 64-bit fixed-point sums (scale
2^28).  Integer sums add exactly and in any order, so one all-reduce (SUM)
over the process group — NCCL over NVLink for device tensors, gloo for host
tensors — yields the single-device sums, and :func:`resolve_sums` turns them
into the image with the arithmetic of the device resolve (sum converted to
double, times 1 / (2^28 * spp) in double, rounded to float32).  The result
equals the single-device ``render_frame`` of the same frame bit for bit on
every rank.  The reduction is the frame's one exchange step: 24 bytes per
pixel per rank (50 MB for 1080p).
"""

from __future__ import annotations

import numpy as np

ACCUM_SCALE = 268435456.0   # 2^28, the device accumulator's fixed-point scale
SAMPLE_CLAMP = 524287.0     # 2^19 - 1, the device's per-sample clamp of each channel
MAX_FRAME_SAMPLES = 65536   # samples of one frame, over all shards: sums stay below 2^63


def sample_shard(samples: int, world: int, rank: int) -> tuple[int, int]:
    """(first sample, count) of rank `rank`: contiguous, as even as possible,
    covering [0, samples) exactly once over the ranks."""
    samples, world, rank = int(samples), int(world), int(rank)
    if samples < 1 or world < 1 or not 0 <= rank < world:
        raise ValueError("samples and world must be positive and rank in [0, world)")
    base, extra = divmod(samples, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def resolve_sums(sums, samples: int):
    """Image (h, w, 4) float32 from fixed-point sums (h, w, 3) of `samples`
    samples: numpy arrays give numpy, torch tensors give torch on their
    device."""
    scale = 1.0 / (ACCUM_SCALE * float(samples))
    if hasattr(sums, "double"):
        import torch

        rgb = (sums.to(torch.float64) * scale).to(torch.float32)
        return torch.cat([rgb, torch.zeros_like(rgb[..., :1])], dim=-1)
    sums = np.asarray(sums)
    if sums.dtype.kind == "i" and np.any(sums < 0):
        raise ValueError("fixed-point sums cannot be negative")
    rgb = (sums.astype(np.uint64).astype(np.float64) * scale).astype(np.float32)
    return np.concatenate([rgb, np.zeros(rgb.shape[:-1] + (1,), np.float32)], axis=-1)


def render_frame_sharded(renderer, scene, camera, width: int, height: int, *, samples=None, frame_index: int = 0,
                         max_bounces=None, group=None):
    """Render one frame with its samples split over the ranks of `group`
    (torch.distributed's default group when None) and return the image on
    every rank.  `renderer` is this rank's CudaWavefrontRenderer."""
    import torch
    import torch.distributed as dist

    from .renderers.cuda import RenderRequest

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    spp = renderer.config.samples_per_pixel if samples is None else int(samples)
    if not 1 <= spp <= MAX_FRAME_SAMPLES:
        # the signed 64-bit all-reduce stays exact only up to this many samples per pixel
        raise ValueError(f"samples must be between 1 and {MAX_FRAME_SAMPLES}")
    first, count = sample_shard(spp, world, rank)
    device = torch.device(renderer.device)
    sums = torch.zeros((int(height), int(width), 3), dtype=torch.int64, device=device)
    if count:
        image = torch.empty((int(height), int(width), 4), dtype=torch.float32, device=device)
        renderer.render_batch([RenderRequest(scene, camera, width, height, samples=count, frame_index=frame_index,
                                             max_bounces=max_bounces, first_sample=first)],
                              outs=[image], sums=[sums])
    if world > 1:
        dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    return resolve_sums(sums, spp)


__all__ = ["ACCUM_SCALE", "SAMPLE_CLAMP", "MAX_FRAME_SAMPLES", "sample_shard", "resolve_sums", "render_frame_sharded"]
